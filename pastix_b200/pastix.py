"""Python interface mirroring PaStiX's ``pypastix`` wrapper
(wrappers/python/examples/pypastix/pastix.py, __pastix__.py:136-383):
``initParam``, ``init``, ``task_analyze``, ``task_numfact``, ``task_solve``,
``task_refine``, ``finalize`` and the ``solver`` class, same argument
meaning, with errors raised as :class:`PastixError` carrying the reference's
error codes.
"""
from __future__ import annotations

import ctypes as C
from enum import IntEnum

import numpy as np

from . import _lib
from ._lib import PDBL, PINT, pastix_int_t, pastix_order_t, pgpu_solver_info_t
from .spm import mtxtype, spmatrix


class iparm(IntEnum):
    verbose = 0; io_strategy = 1; nnzeros = 2; nnzeros_block_local = 3; allocated_terms = 4
    produce_stats = 5; trace = 6; mc64 = 7; ordering = 8; ordering_default = 9
    min_blocksize = 36; max_blocksize = 37; tasks2d_level = 38; tasks2d_width = 39; allcand = 40
    incomplete = 41; level_of_fill = 42; factorization = 43; facto_look_side = 44; static_pivoting = 45
    free_cscuser = 46; schur_fact_mode = 47; transpose_solve = 48; schur_solv_mode = 49; applyperm_ws = 50
    refinement = 51; nbiter = 52; itermax = 53; gmres_im = 54; scheduler = 55; thread_nbr = 56
    gpu_nbr = 59; mixed = 71; ftz = 72; mpi_thread_level = 73; modify_parameter = 74; start_task = 75
    end_task = 76; float_ = 77; mtx_type = 78; dof_nbr = 79; size = 80


class dparm(IntEnum):
    fill_in = 0; epsilon_refinement = 1; relative_error = 2; epsilon_magn_ctrl = 3; order_time = 4
    symbfact_time = 5; reorder_time = 6; blend_time = 7; analyze_time = 8; pred_fact_time = 9
    fact_time = 10; fact_flops = 11; fact_thflops = 12; fact_rlflops = 13; fact_energy = 14
    mem_fr = 15; mem_lr = 16; solv_time = 17; solv_flops = 18; solv_thflops = 19; solv_rlflops = 20
    solv_energy = 21; refine_time = 22; a_norm = 23; compress_tolerance = 24; compress_min_ratio = 25; size = 26


class factotype(IntEnum):
    POTRF = 0; SYTRF = 1; GETRF = 2; PXTRF = 3; HETRF = 4
    LLH = 0; LDLT = 1; LU = 2; LLT = 3; LDLH = 4


class io(IntEnum):
    No = 0; Load = 1; Save = 2; LoadGraph = 4; SaveGraph = 8; LoadCSC = 16; SaveCSC = 32


class refine(IntEnum):
    GMRES = 0; CG = 1; SR = 2; BiCGSTAB = 3


class ordering(IntEnum):
    Scotch = 0; Metis = 1; Personal = 2; PtScotch = 3; ParMetis = 4


class verbose(IntEnum):
    Not = 0; No = 1; Yes = 2


class error(IntEnum):
    SUCCESS = 0; UNKNOWN = 1; ALLOC = 2; NOTIMPLEMENTED = 3; OUTOFMEMORY = 4; THREAD = 5
    INTERNAL = 6; BADPARAMETER = 7; FILE = 8; INTEGER_TYPE = 9; IO = 10; MPI = 11


class PastixError(RuntimeError):
    def __init__(self, func: str, code: int):
        try:
            name = error(code).name
        except ValueError:
            name = str(code)
        super().__init__(f"{func} returned PASTIX_ERR_{name} ({code})")
        self.code = code


def _check(func: str, rc: int) -> None:
    if rc != 0:
        raise PastixError(func, rc)


assert int(iparm.size) == 80 and int(dparm.size) == 26


class Data:
    """Owner of an opaque ``pastix_data_t*`` plus the iparm/dparm arrays it points to."""

    def __init__(self, ptr: C.c_void_p, ip: np.ndarray, dp: np.ndarray):
        self.ptr = ptr
        self.iparm = ip
        self.dparm = dp
        self._keep: list = []

    def __del__(self):
        try:
            finalize(self)
        except Exception:
            pass


def initParam():
    """pastixInitParam: returns (iparm, dparm) numpy arrays with the defaults."""
    lib = _lib.load()
    ip = np.zeros(int(iparm.size), dtype=np.int64)
    dp = np.zeros(int(dparm.size), dtype=np.float64)
    lib.pastixInitParam(ip.ctypes.data_as(PINT), dp.ctypes.data_as(PDBL))
    return ip, dp


def init(ip: np.ndarray, dp: np.ndarray) -> Data:
    lib = _lib.load()
    p = C.c_void_p()
    lib.pastixInit(C.byref(p), 0, ip.ctypes.data_as(PINT), dp.ctypes.data_as(PDBL))
    if not p:
        raise PastixError("pastixInit", int(error.BADPARAMETER))
    return Data(p, ip, dp)


def finalize(pd: Data) -> None:
    if pd.ptr:
        _lib.load().pastixFinalize(C.byref(pd.ptr))
        pd.ptr = C.c_void_p()


def orderGrid(nx: int, ny: int, nz: int):
    """pastixOrderGrid: returns (permtab, peritab, rangtab, treetab) as numpy arrays."""
    lib = _lib.load()
    o = pastix_order_t()
    po = C.pointer(o)
    _check("pastixOrderGrid", lib.pastixOrderGrid(C.byref(po), nx, ny, nz))
    n, cb = o.vertnbr, o.cblknbr
    res = tuple(np.ctypeslib.as_array(a, shape=(s,)).copy()
                for a, s in ((o.permtab, n), (o.peritab, n), (o.rangtab, cb + 1), (o.treetab, cb)))
    lib.pastixOrderExit(C.byref(o))
    return res


def orderLoad(pd: Data = None):
    """pastixOrderLoad: the ordering file ($PASTIX_FILE_ORDER or "ordername") as
    (permtab, peritab, rangtab, treetab) numpy arrays (treetab None for a
    version-0 file, which has no elimination tree)."""
    lib = _lib.load()
    o = pastix_order_t()
    _check("pastixOrderLoad", lib.pastixOrderLoad(pd.ptr if pd is not None else None, C.byref(o)))
    n, cb = o.vertnbr, o.cblknbr
    get = lambda a, s: np.ctypeslib.as_array(a, shape=(s,)).copy() if a else None  # noqa: E731
    res = (get(o.permtab, n), get(o.peritab, n), get(o.rangtab, cb + 1), get(o.treetab, cb))
    lib.pastixOrderExit(C.byref(o))
    return res


def subtask_order(pd: Data, spm: spmatrix, perm=None, rangtab=None, treetab=None) -> None:
    """pastix_subtask_order with an optional personal ordering (iparm ordering = Personal)."""
    lib = _lib.load()
    po = None
    if perm is not None:
        perm = np.ascontiguousarray(perm, dtype=np.int64)
        peri = np.empty_like(perm)
        peri[perm] = np.arange(perm.size, dtype=np.int64)
        o = pastix_order_t()
        o.baseval = 0
        o.vertnbr = perm.size
        o.permtab = perm.ctypes.data_as(PINT)
        o.peritab = peri.ctypes.data_as(PINT)
        keep = [perm, peri]
        if rangtab is not None and treetab is not None:
            rangtab = np.ascontiguousarray(rangtab, dtype=np.int64)
            treetab = np.ascontiguousarray(treetab, dtype=np.int64)
            o.cblknbr = rangtab.size - 1
            o.rangtab = rangtab.ctypes.data_as(PINT)
            o.treetab = treetab.ctypes.data_as(PINT)
            keep += [rangtab, treetab]
        pd._keep = keep
        po = C.byref(o)
        pd.iparm[iparm.ordering] = ordering.Personal
    _check("pastix_subtask_order", lib.pastix_subtask_order(pd.ptr, spm.pointer(), po))


def subtask_symbfact(pd: Data) -> None:
    _check("pastix_subtask_symbfact", _lib.load().pastix_subtask_symbfact(pd.ptr))


def subtask_reordering(pd: Data) -> None:
    _check("pastix_subtask_reordering", _lib.load().pastix_subtask_reordering(pd.ptr))


def subtask_blend(pd: Data) -> None:
    _check("pastix_subtask_blend", _lib.load().pastix_subtask_blend(pd.ptr))


def task_analyze(pd: Data, spm: spmatrix) -> None:
    _check("pastix_task_analyze", _lib.load().pastix_task_analyze(pd.ptr, spm.pointer()))


def analyze_grid(pd: Data, spm: spmatrix, nx: int, ny: int, nz: int) -> None:
    """The ordering_grid example's analysis: grid nested dissection as a personal
    ordering (example/ordering_grid.c:100-123), then symbfact, reordering, blend.
    A matrix with dof > 1 unknowns per grid node is given expanded; the node
    ordering is expanded by dof."""
    perm, _, rang, tree = orderGrid(nx, ny, nz)
    subtask_order(pd, spm, perm, rang, tree)
    subtask_symbfact(pd)
    subtask_reordering(pd)
    subtask_blend(pd)


def set_symbol(pd: Data, spm: spmatrix, permtab, cb_fcol, cb_lcol, cb_fblok, bk_frow, bk_lrow, bk_fcblk) -> None:
    """pgpu_set_symbol: use an ordering + block symbolic structure computed
    elsewhere (e.g. exported from the reference's SolverMatrix)."""
    arrs = [np.ascontiguousarray(a, dtype=np.int64) for a in (permtab, cb_fcol, cb_lcol, cb_fblok, bk_frow, bk_lrow,
                                                               bk_fcblk)]
    pd._keep = arrs
    p = [a.ctypes.data_as(PINT) for a in arrs]
    _check("pgpu_set_symbol", _lib.load().pgpu_set_symbol(pd.ptr, spm.pointer(), p[0], len(arrs[1]), p[1], p[2], p[3],
                                                           len(arrs[4]), p[4], p[5], p[6]))


def task_numfact(pd: Data, spm: spmatrix) -> None:
    _check("pastix_task_numfact", _lib.load().pastix_task_numfact(pd.ptr, spm.pointer()))


def task_solve(pd: Data, spm: spmatrix, x: np.ndarray) -> None:
    """Solve in place: x holds b on entry (n or n x nrhs, Fortran order)."""
    if not (x.dtype == np.float64 and (x.flags.f_contiguous or x.ndim == 1)):
        raise ValueError("x must be a float64 Fortran-ordered array")
    nrhs = 1 if x.ndim == 1 else x.shape[1]
    n = x.shape[0]
    _check("pastix_task_solve", _lib.load().pastix_task_solve(pd.ptr, n, nrhs, x.ctypes.data, n))


def task_refine(pd: Data, spm: spmatrix, b: np.ndarray, x: np.ndarray) -> None:
    nrhs = 1 if x.ndim == 1 else x.shape[1]
    n = x.shape[0]
    b = np.asfortranarray(b, dtype=np.float64)
    _check("pastix_task_refine",
           _lib.load().pastix_task_refine(pd.ptr, n, nrhs, b.ctypes.data, n, x.ctypes.data, n))


def solver_info(pd: Data) -> dict:
    """Structure of the analysed problem as numpy arrays (copies)."""
    info = pgpu_solver_info_t()
    _check("pgpu_solver_info", _lib.load().pgpu_solver_info(pd.ptr, C.byref(info)))
    cb, bk = info.cblknbr, info.bloknbr

    def arr(p, s):
        return np.ctypeslib.as_array(p, shape=(s,)).copy() if s > 0 else np.zeros(0, np.int64)

    return dict(n=info.n, cblknbr=cb, bloknbr=bk, coefnbr=info.coefnbr, nlevels=info.nlevels,
                ntasks=info.ntasks, thflops=info.thflops,
                cb_fcol=arr(info.cb_fcol, cb), cb_lcol=arr(info.cb_lcol, cb), cb_fblok=arr(info.cb_fblok, cb + 1),
                cb_stride=arr(info.cb_stride, cb), cb_coef=arr(info.cb_coef, cb + 1), cb_level=arr(info.cb_level, cb),
                bk_frow=arr(info.bk_frow, bk), bk_lrow=arr(info.bk_lrow, bk), bk_fcblk=arr(info.bk_fcblk, bk),
                bk_lcblk=arr(info.bk_lcblk, bk), bk_rowoff=arr(info.bk_rowoff, bk),
                permtab=arr(info.permtab, info.n), peritab=arr(info.peritab, info.n))


def get_coeftab(pd: Data, with_u: bool = False):
    """Factor panels in the library layout (L, U or None)."""
    info = solver_info(pd)
    dt = np.float32 if pd.iparm[iparm.mixed] else np.float64
    L = np.empty(max(1, info["coefnbr"]), dtype=dt)
    U = np.empty_like(L) if with_u else None
    _check("pgpu_get_coeftab", _lib.load().pgpu_get_coeftab(pd.ptr, L.ctypes.data, U.ctypes.data if with_u else None))
    return L, U


class solver:
    """Object interface (wrappers/python/examples/pypastix/solver.py:21-200)."""

    def __init__(self, A=None, **kwargs):
        self.iparm, self.dparm = initParam()
        self.verbose = kwargs.setdefault("verbose", verbose.Not)
        self.iparm[iparm.verbose] = int(self.verbose)
        self.mtxtype = kwargs.setdefault("mtxtype", mtxtype.General)
        ft = factotype.LU
        if self.mtxtype == mtxtype.Symmetric:
            ft = factotype.LDLT
        self.factotype = kwargs.setdefault("factotype", ft)
        self.iparm[iparm.factorization] = int(self.factotype)
        if kwargs.get("mixed"):
            self.iparm[iparm.mixed] = 1
        self.pastix_data = init(self.iparm, self.dparm)
        self.grid = kwargs.get("grid")
        if A is not None:
            self.setup(A)

    def setup(self, A):
        self.A = A
        st = mtxtype.Symmetric if self.factotype in (factotype.LLT, factotype.POTRF, factotype.LDLT) else mtxtype.General
        self.spmA = spmatrix(A, st)
        if self.grid is not None:
            analyze_grid(self.pastix_data, self.spmA, *self.grid)
        else:
            task_analyze(self.pastix_data, self.spmA)
        task_numfact(self.pastix_data, self.spmA)

    def solve(self, b, refine=True):
        x = np.asfortranarray(b, dtype=np.float64).copy(order="F")
        task_solve(self.pastix_data, self.spmA, x)
        if refine:
            task_refine(self.pastix_data, self.spmA, b, x)
        return x

    def finalize(self):
        finalize(self.pastix_data)


# ---------------- device-resident entry points (torch CUDA tensors) ----------------
def stream_ptr(pd: Data) -> int:
    """cudaStream_t of the library (after the analysis)."""
    p = _lib.load().pgpu_stream(pd.ptr)
    if not p:
        raise PastixError("pgpu_stream", int(error.INTERNAL))
    return int(p)


def _torch_stream():
    import torch
    return torch.cuda.current_stream()


def numfact_device(pd: Data, values) -> None:
    """Numerical factorization from a CUDA float64 tensor of the spm values
    (the caller's stream is synchronised first: the library works on its own stream)."""
    _torch_stream().synchronize()
    _check("pgpu_numfact_device", _lib.load().pgpu_numfact_device(pd.ptr, C.c_void_p(values.data_ptr())))


def _ld(B) -> int:
    """Leading dimension of a column-major n or n x nrhs CUDA tensor (the
    stride of a single column is arbitrary in torch, so it is not read)."""
    if B.dim() == 1 or B.shape[1] == 1:
        if B.dim() == 2 and B.stride(0) != 1 and B.shape[0] > 1:
            raise ValueError("right-hand sides must be column major (unit stride down a column)")
        return B.shape[0]
    if B.stride(0) != 1:
        raise ValueError("right-hand sides must be column major (unit stride down a column)")
    return B.stride(1)


def solve_device(pd: Data, B, transposed: bool = False) -> None:
    """In-place solve of a CUDA float64 tensor B (n or n x nrhs, column-major storage)."""
    n = B.shape[0]
    nrhs = 1 if B.dim() == 1 else B.shape[1]
    ld = _ld(B)
    fn = _lib.load().pgpu_solve_transposed_device if transposed else _lib.load().pgpu_solve_device
    _check("pgpu_solve_device", fn(pd.ptr, nrhs, C.c_void_p(B.data_ptr()), ld,
                                   C.c_void_p(_torch_stream().cuda_stream)))


def solve_refine_device(pd: Data, B, X) -> None:
    """X <- refined solution of A X = B (CUDA float64 tensors, column-major)."""
    nrhs = 1 if B.dim() == 1 else B.shape[1]
    ldb, ldx = _ld(B), _ld(X)
    _torch_stream().synchronize()
    _check("pgpu_solve_refine_device",
           _lib.load().pgpu_solve_refine_device(pd.ptr, nrhs, C.c_void_p(B.data_ptr()), ldb,
                                                C.c_void_p(X.data_ptr()), ldx))


def spmv_device(pd: Data, alpha: float, x, beta: float, y) -> None:
    _check("pgpu_spmv_device", _lib.load().pgpu_spmv_device(pd.ptr, alpha, C.c_void_p(x.data_ptr()), beta,
                                                            C.c_void_p(y.data_ptr()),
                                                            C.c_void_p(_torch_stream().cuda_stream)))


def set_tuning(pd: Data, dmma_n: int, dmma_k: int, tc_k: int) -> None:
    """Bucket boundaries of the update tiles (see pgpu_set_tuning)."""
    _check("pgpu_set_tuning", _lib.load().pgpu_set_tuning(pd.ptr, dmma_n, dmma_k, tc_k))


def get_tuning(pd: Data) -> tuple:
    v = np.zeros(3, dtype=np.int64)
    _check("pgpu_get_tuning", _lib.load().pgpu_get_tuning(pd.ptr, v.ctypes.data_as(PINT)))
    return tuple(int(x) for x in v)


def autotune(pd: Data, values) -> tuple:
    """Time the candidate update-tile buckets on factorizations of `values` (CUDA
    float64 tensor, spm order); the fastest stays in effect.  Returns
    (dmma_n, dmma_k, tc_k)."""
    _torch_stream().synchronize()
    v = np.zeros(3, dtype=np.int64)
    _check("pgpu_autotune", _lib.load().pgpu_autotune(pd.ptr, C.c_void_p(values.data_ptr()), v.ctypes.data_as(PINT)))
    return tuple(int(x) for x in v)


def refine_block(pd: Data, enable: bool) -> None:
    """GMRES refinement of several right-hand sides as one block (default on)."""
    _check("pgpu_refine_block", _lib.load().pgpu_refine_block(pd.ptr, int(enable)))


def graphs(pd: Data, enable: bool) -> None:
    """Replay the factorization and solve launch sequences as CUDA graphs (default on)."""
    _check("pgpu_graphs", _lib.load().pgpu_graphs(pd.ptr, int(enable)))


def profile(pd: Data, enable: bool) -> None:
    _check("pgpu_profile", _lib.load().pgpu_profile(pd.ptr, int(enable)))


def profile_get(pd: Data) -> dict:
    """{class: (device ms, launches)} accumulated since the last profile() call."""
    k = len(_lib.PROFILE_CLASSES)
    ms = np.zeros(k, dtype=np.float64)
    ln = np.zeros(k, dtype=np.int64)
    _check("pgpu_profile_get", _lib.load().pgpu_profile_get(pd.ptr, ms.ctypes.data_as(PDBL),
                                                            ln.ctypes.data_as(C.POINTER(C.c_longlong)), k))
    return {c: (float(ms[i]), int(ln[i])) for i, c in enumerate(_lib.PROFILE_CLASSES)}
