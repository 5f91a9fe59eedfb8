"""Error returns of the C ABI that need no GPU: malformed plan descriptions give
DMRGB200_INVALID_PLAN with a message (the reference's builders throw
std::runtime_error and its executors exit the process instead), and the
allocation-free H·psi rejects plans larger than its static area before touching
the device.  Plans are built by hand here so that each check flips one field."""
import ctypes as C

import numpy as np
import pytest

from dmrgb200 import _capi as capi


def one_task_plan(ls=8, rs=8, nb=2):
    """A minimal valid H·psi plan: one input block (ls x rs), one output block of the
    same shape, one T task reading the whole block against a cohort of nb blocks
    (rs x rs), one cohort with one unit whose single line has one term."""
    u = lambda *v: np.array(v, dtype=np.uint32)
    return {
        "kind": capi.PLAN_HPSI, "in_size": ls * rs, "out_size": ls * rs,
        "g_t": u(0, 1), "g_c": u(0, 1),
        "in_rows": u(ls), "in_cols": u(rs), "in_off": np.array([0], np.uint64),
        "out_rows": u(ls), "out_cols": u(rs), "out_off": np.array([0], np.uint64),
        "t_lb": u(0), "t_col": u(0), "t_ci": u(0), "t_trans": np.zeros(1, np.uint8), "t_nb": u(nb),
        "t_brows": u(rs), "t_bcols": u(rs), "t_width": u(),
        "c_lb": u(0), "c_rb": u(0), "c_ls": u(ls), "c_rs": u(ls), "c_ci": u(0), "c_trans": np.zeros(1, np.uint8),
        "c_nsrows": u(1), "c_stripe": u(rs), "c_out_ci": u(0), "c_unit": u(0, 1),
        "u_offset": u(0), "u_ms": u(rs), "u_line": u(0, 1),
        "l_b1": u(0), "l_term": u(0, 1),
        "term_alpha": np.ones(1), "term_t": u(0), "term_col": u(0),
    }


def validate(plan):
    desc, keep = capi.numpy_to_desc(plan)
    st = capi.lib.dmrgb200_plan_validate(C.byref(desc))
    msg = capi.lib.dmrgb200_last_error().decode()
    del keep
    return st, msg


def test_minimal_plan_is_valid():
    st, msg = validate(one_task_plan())
    assert st == capi.OK, msg


@pytest.mark.parametrize("field,value,words", [
    ("term_t", [5], "T task of another group"),
    ("t_col", [3], "column slice exceeds block"),
    ("l_b1", [4], "row block out of range"),
    ("term_col", [20], "past T columns"),
    ("u_offset", [2], "unit exceeds stripe"),
    ("c_stripe", [4], ""),
    ("l_term", [0, 2], "do not cover the terms"),
    ("g_t", [0, 0], "do not cover"),
])
def test_malformed_plans_are_rejected(field, value, words):
    plan = one_task_plan()
    plan[field] = np.array(value, dtype=plan[field].dtype)
    st, msg = validate(plan)
    assert st == 2, (field, st, msg)  # DMRGB200_INVALID_PLAN
    assert words in msg, msg


def test_noalloc_rejects_plans_beyond_its_static_area():
    """T alone needs ls x nb x rs doubles = 1024 x 8 x 1024 x 8 B = 64 MiB, so the plan
    cannot fit the 64 MiB area; the call must say so (with the size) before it
    looks up or touches any device memory, so this runs without a GPU.  The
    boundary 'pointers' are placeholders that the rejected call never reads."""
    plan = one_task_plan(ls=1024, rs=1024, nb=8)
    desc, keep = capi.numpy_to_desc(plan)
    fake = (C.c_void_p * 1)(0x1000)
    view = capi.BoundaryView()
    view.n_cohorts = 1
    view.cohort_ptr = C.cast(fake, C.POINTER(C.c_void_p))
    st = capi.lib.dmrgb200_hpsi_noalloc(C.byref(desc), C.byref(view), C.byref(view), 0x2000, 0x3000, None)
    msg = capi.lib.dmrgb200_last_error().decode()
    assert st == 3, (st, msg)  # DMRGB200_OUT_OF_MEMORY
    assert "bytes of scratch" in msg and str(64 << 20) in msg, msg
    del keep


def test_library_exports_every_declared_entry_point():
    """Every function include/dmrgb200.h declares is exported by libdmrgb200.so and has
    a ctypes signature in the binding (loading needs no GPU)."""
    import ctypes
    import re
    from pathlib import Path

    header = (Path(__file__).resolve().parent.parent / "include" / "dmrgb200.h").read_text()
    names = set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\*?(dmrgb200_\w+)\s*\(", header, re.M))
    assert len(names) > 40, names
    lib = ctypes.CDLL(str(capi.LIB_PATH))
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    unbound = [n for n in sorted(names) if n not in capi.EXPORTED]
    assert not unbound, unbound
