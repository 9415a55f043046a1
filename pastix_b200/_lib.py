"""ctypes binding of ``libpastix_b200.so`` (the C ABI of include/pastix_b200.h).

The library is built in-tree by :mod:`pastix_b200.build`; loading it needs the
CUDA runtime but no GPU (analysis entry points run on the host).  Numerical
entry points return ``PASTIX_ERR_INTERNAL`` when no CUDA device is present:
there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libpastix_b200.so"

pastix_int_t = C.c_int64
PINT = C.POINTER(pastix_int_t)
PDBL = C.POINTER(C.c_double)
VP = C.c_void_p

# names declared in include/pastix_b200.h (checked by the CPU test-suite)
EXPORTS = [
    "pastixInitParam", "pastixInit", "pastixInitWithAffinity", "pastixFinalize",
    "pastix_task_analyze", "pastix_task_numfact", "pastix_task_solve", "pastix_task_refine",
    "pastix_task_solve_and_refine", "pastix",
    "pastix_subtask_order", "pastix_subtask_symbfact", "pastix_subtask_reordering", "pastix_subtask_blend",
    "pastix_subtask_spm2bcsc", "pastix_subtask_bcsc2ctab", "pastix_subtask_sopalin",
    "pastix_subtask_applyorder", "pastix_subtask_trsm", "pastix_subtask_diag", "pastix_subtask_solve",
    "pastix_subtask_solve_adv", "pastix_subtask_refine",
    "pastixRhsInit", "pastixRhsFinalize", "pastixRhsDoubletoSingle", "pastixRhsSingleToDouble",
    "pastixOrderGrid", "pastixOrderExit", "pastixOrderLoad", "pastixOrderSave",
    "pgpu_solver_info", "pgpu_get_coeftab", "pgpu_solve_device", "pgpu_solve_transposed_device",
    "pgpu_numfact_device", "pgpu_sampled_outer", "pgpu_spmv_device", "pgpu_device_status",
    "pgpu_stream", "pgpu_solve_refine_device", "pgpu_profile", "pgpu_profile_get", "pgpu_set_symbol",
    "pgpu_solve_device_static", "pgpu_graphs", "pgpu_set_tuning", "pgpu_get_tuning", "pgpu_autotune",
    "pgpu_refine_block", "pgpu_wait_selftest",
]

# kernel classes of pgpu_profile_get, in order
PROFILE_CLASSES = ["fill", "panel_small", "diag_large", "trsm", "update", "fwd_diag", "fwd_update",
                   "bwd_update", "bwd_diag", "spmv", "vec", "update_big", "split"]


class spmatrix_t(C.Structure):
    _fields_ = [
        ("mtxtype", C.c_int), ("flttype", C.c_int), ("fmttype", C.c_int),
        ("baseval", pastix_int_t), ("gN", pastix_int_t), ("n", pastix_int_t),
        ("gnnz", pastix_int_t), ("nnz", pastix_int_t),
        ("gNexp", pastix_int_t), ("nexp", pastix_int_t), ("gnnzexp", pastix_int_t), ("nnzexp", pastix_int_t),
        ("dof", pastix_int_t), ("dofs", PINT), ("layout", C.c_int),
        ("colptr", PINT), ("rowptr", PINT), ("loc2glob", PINT), ("values", VP), ("glob2loc", PINT),
        ("clustnum", C.c_int), ("clustnbr", C.c_int), ("comm", C.c_int), ("replicated", C.c_int),
    ]


class pastix_order_t(C.Structure):
    _fields_ = [
        ("baseval", pastix_int_t), ("vertnbr", pastix_int_t), ("cblknbr", pastix_int_t),
        ("permtab", PINT), ("peritab", PINT), ("rangtab", PINT), ("treetab", PINT),
        ("selevtx", C.POINTER(C.c_int8)), ("sndenbr", pastix_int_t), ("sndetab", PINT),
        ("peritab_exp", PINT),
    ]


class pgpu_solver_info_t(C.Structure):
    _fields_ = [
        ("n", pastix_int_t), ("cblknbr", pastix_int_t), ("bloknbr", pastix_int_t),
        ("coefnbr", pastix_int_t), ("nlevels", pastix_int_t), ("ntasks", pastix_int_t),
        ("cb_fcol", PINT), ("cb_lcol", PINT), ("cb_fblok", PINT), ("cb_stride", PINT),
        ("cb_coef", PINT), ("cb_level", PINT),
        ("bk_frow", PINT), ("bk_lrow", PINT), ("bk_fcblk", PINT), ("bk_lcblk", PINT), ("bk_rowoff", PINT),
        ("permtab", PINT), ("peritab", PINT),
        ("thflops", C.c_double),
    ]


_lib = None


def load() -> C.CDLL:
    """Load the shared library (once) and declare the prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run `python -m pastix_b200.build` first")
    lib = C.CDLL(str(LIB_PATH))
    P = VP  # opaque pointers
    proto = {
        "pastixInitParam": (None, [PINT, PDBL]),
        "pastixInit": (None, [C.POINTER(P), C.c_int, PINT, PDBL]),
        "pastixFinalize": (None, [C.POINTER(P)]),
        "pastix_task_analyze": (C.c_int, [P, C.POINTER(spmatrix_t)]),
        "pastix_task_numfact": (C.c_int, [P, C.POINTER(spmatrix_t)]),
        "pastix_task_solve": (C.c_int, [P, pastix_int_t, pastix_int_t, VP, pastix_int_t]),
        "pastix_task_refine": (C.c_int, [P, pastix_int_t, pastix_int_t, VP, pastix_int_t, VP, pastix_int_t]),
        "pastix_task_solve_and_refine": (C.c_int, [P, pastix_int_t, pastix_int_t, VP, pastix_int_t, VP, pastix_int_t]),
        "pastix": (C.c_int, [C.POINTER(P), C.c_int, pastix_int_t, PINT, PINT, VP, PINT, PINT, VP, pastix_int_t,
                             PINT, PDBL]),
        "pastix_subtask_order": (C.c_int, [P, C.POINTER(spmatrix_t), C.POINTER(pastix_order_t)]),
        "pastix_subtask_symbfact": (C.c_int, [P]),
        "pastix_subtask_reordering": (C.c_int, [P]),
        "pastix_subtask_blend": (C.c_int, [P]),
        "pastix_subtask_spm2bcsc": (C.c_int, [P, C.POINTER(spmatrix_t)]),
        "pastix_subtask_bcsc2ctab": (C.c_int, [P]),
        "pastix_subtask_sopalin": (C.c_int, [P]),
        "pastix_subtask_applyorder": (C.c_int, [P, C.c_int, pastix_int_t, pastix_int_t, VP, pastix_int_t, P]),
        "pastix_subtask_trsm": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.c_int, P]),
        "pastix_subtask_diag": (C.c_int, [P, P]),
        "pastix_subtask_solve": (C.c_int, [P, P]),
        "pastix_subtask_solve_adv": (C.c_int, [P, C.c_int, P]),
        "pastix_subtask_refine": (C.c_int, [P, P, P]),
        "pastixRhsInit": (C.c_int, [C.POINTER(P)]),
        "pastixRhsFinalize": (C.c_int, [P]),
        "pastixOrderGrid": (C.c_int, [C.POINTER(C.POINTER(pastix_order_t)), pastix_int_t, pastix_int_t, pastix_int_t]),
        "pastixOrderExit": (None, [C.POINTER(pastix_order_t)]),
        "pastixOrderLoad": (C.c_int, [P, C.POINTER(pastix_order_t)]),
        "pastixOrderSave": (C.c_int, [P, C.POINTER(pastix_order_t)]),
        "pgpu_solver_info": (C.c_int, [P, C.POINTER(pgpu_solver_info_t)]),
        "pgpu_get_coeftab": (C.c_int, [P, VP, VP]),
        "pgpu_solve_device": (C.c_int, [P, pastix_int_t, VP, pastix_int_t, VP]),
        "pgpu_solve_device_static": (C.c_int, [P, pastix_int_t, VP, pastix_int_t, VP]),
        "pgpu_solve_transposed_device": (C.c_int, [P, pastix_int_t, VP, pastix_int_t, VP]),
        "pgpu_numfact_device": (C.c_int, [P, VP]),
        "pgpu_sampled_outer": (C.c_int, [P, C.c_double, VP, VP, VP, VP]),
        "pgpu_spmv_device": (C.c_int, [P, C.c_double, VP, C.c_double, VP, VP]),
        "pgpu_device_status": (C.c_int, [P]),
        "pgpu_wait_selftest": (C.c_int, [C.POINTER(C.c_int)]),
        "pgpu_stream": (C.c_void_p, [P]),
        "pgpu_solve_refine_device": (C.c_int, [P, pastix_int_t, VP, pastix_int_t, VP, pastix_int_t]),
        "pgpu_profile": (C.c_int, [P, C.c_int]),
        "pgpu_graphs": (C.c_int, [P, C.c_int]),
        "pgpu_refine_block": (C.c_int, [P, C.c_int]),
        "pgpu_set_tuning": (C.c_int, [P, pastix_int_t, pastix_int_t, pastix_int_t]),
        "pgpu_get_tuning": (C.c_int, [P, PINT]),
        "pgpu_autotune": (C.c_int, [P, VP, PINT]),
        "pgpu_profile_get": (C.c_int, [P, PDBL, C.POINTER(C.c_longlong), C.c_int]),
        "pgpu_set_symbol": (C.c_int, [P, C.POINTER(spmatrix_t), PINT, pastix_int_t, PINT, PINT, PINT, pastix_int_t,
                                      PINT, PINT, PINT]),
    }
    for name, (res, args) in proto.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
