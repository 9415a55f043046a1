"""Analysis files (IPARM_IO_STRATEGY): the ordering and the block symbolic
matrix written in the reference's text formats (order/order_io.c,
symbol/symbol_io.c) by PastixIOSave, read back by PastixIOLoad into an
identical analysis, and a hand-written reference-format ordering file read by
pastixOrderLoad.  Host only."""
from __future__ import annotations

import glob
import os
import shutil

import numpy as np

from pastix_b200 import gen
from pastix_b200 import pastix as px
from pastix_b200.spm import mtxtype, spmatrix

KEYS = ("permtab", "cb_fcol", "cb_lcol", "cb_fblok", "bk_frow", "bk_lrow", "bk_fcblk", "cb_stride")


def _analyze(A, io=px.io.No, ordering=None):
    ip, dp = px.initParam()
    ip[px.iparm.io_strategy] = int(io)
    if ordering is not None:
        ip[px.iparm.ordering] = int(ordering)
    pd = px.init(ip, dp)
    S = spmatrix(A, mtxtype.Symmetric)
    px.task_analyze(pd, S)
    return pd, px.solver_info(pd)


def _ints(path):
    with open(path) as f:
        return [int(t) for t in f.read().split()]


def test_save_then_load_gives_the_same_analysis(lib, tmp_path, monkeypatch):
    A = gen.laplacian7(9, 8, 7)
    n = A.shape[0]
    monkeypatch.setenv("PASTIX_OUTPUT_DIR", str(tmp_path / "pastix"))
    monkeypatch.delenv("PASTIX_FILE_ORDER", raising=False)
    pd, ref = _analyze(A, io=px.io.Save)
    dirs = glob.glob(str(tmp_path / "pastix-*"))
    assert len(dirs) == 1
    order = _ints(os.path.join(dirs[0], "ordergen"))
    symb = _ints(os.path.join(dirs[0], "symbgen"))
    # ordering file: version 1, cblknbr, vertnbr, rangtab, permtab, treetab
    assert order[0] == 1 and order[2] == n
    cb = order[1]
    assert len(order) == 3 + (cb + 1) + n + cb
    rang = np.array(order[3:4 + cb])
    perm = np.array(order[4 + cb:4 + cb + n])
    tree = np.array(order[4 + cb + n:])
    assert rang[0] == 0 and rang[-1] == n and np.all(np.diff(rang) > 0)
    assert np.array_equal(perm, ref["permtab"])
    assert tree[-1] == -1
    # symbol file: version 1, cblknbr, bloknbr, nodenbr, baseval, 3 ints per cblk and per blok
    assert symb[0] == 1 and symb[3] == n and symb[4] == 0
    assert len(symb) == 5 + 3 * (symb[1] + symb[2])
    # load both into a new instance: the same analysis, solver structure included
    shutil.copy(os.path.join(dirs[0], "symbgen"), tmp_path / "symbname")
    monkeypatch.setenv("PASTIX_FILE_ORDER", os.path.join(dirs[0], "ordergen"))
    monkeypatch.chdir(tmp_path)
    pd2, got = _analyze(A, io=px.io.Load, ordering=px.ordering.Personal)
    for k in KEYS:
        assert np.array_equal(np.asarray(got[k]), np.asarray(ref[k])), k
    assert got["thflops"] == ref["thflops"]


def test_order_load_reference_format(lib, tmp_path, monkeypatch):
    """A version-0 ordering file (no elimination tree) in the layout the
    reference writes: 8 integers per line, tab separated, base 1."""
    path = tmp_path / "ordername"
    # 5 vertices, 2 supernodes {1, 2, 3} and {4, 5}; permtab (base 1) = 3 1 5 2 4
    path.write_text("0\n2\t5\n1\t4\t6\n3\t1\t5\t2\t4\n")
    monkeypatch.setenv("PASTIX_FILE_ORDER", str(path))
    perm, peri, rang, tree = px.orderLoad()
    assert perm.tolist() == [2, 0, 4, 1, 3]
    assert peri.tolist() == [1, 3, 0, 4, 2]
    # the supernode partition is kept as read (order/order_io.c:80-85), only the tree is absent
    assert rang.tolist() == [0, 3, 5]
    assert tree is None


def test_load_rejects_a_bad_file(lib, tmp_path, monkeypatch):
    path = tmp_path / "ordername"
    path.write_text("1\n2\t4\n0\t2\t4\n0\t0\t1\t2\n1\t-1\n")  # permtab repeats 0
    monkeypatch.setenv("PASTIX_FILE_ORDER", str(path))
    ip, dp = px.initParam()
    ip[px.iparm.io_strategy] = int(px.io.Load)
    ip[px.iparm.ordering] = int(px.ordering.Personal)
    pd = px.init(ip, dp)
    S = spmatrix(gen.laplacian7(2, 2, 1), mtxtype.Symmetric)
    rc = lib.pastix_task_analyze(pd.ptr, S.pointer())
    assert rc == px.error.FILE


def test_load_rejects_a_corrupted_symbol(lib, tmp_path, monkeypatch):
    """A symbol file whose blok faces an earlier cblk is refused with
    PASTIX_ERR_FILE before the supernode split walks it."""
    A = gen.laplacian7(5, 4, 3)
    monkeypatch.setenv("PASTIX_OUTPUT_DIR", str(tmp_path / "pastix"))
    monkeypatch.delenv("PASTIX_FILE_ORDER", raising=False)
    _analyze(A, io=px.io.Save)
    d = glob.glob(str(tmp_path / "pastix-*"))[0]
    symb = _ints(os.path.join(d, "symbgen"))
    cb, bk = symb[1], symb[2]
    cbt = np.array(symb[5:5 + 3 * cb]).reshape(cb, 3)
    bkt = np.array(symb[5 + 3 * cb:]).reshape(bk, 3)
    # first off-diagonal blok of the last cblk that has one: make it face cblk 0
    for k in range(cb - 1, -1, -1):
        lb = cbt[k + 1, 2] if k + 1 < cb else bk
        if lb - cbt[k, 2] > 1:
            bkt[cbt[k, 2] + 1, 2] = 0
            break
    else:
        raise AssertionError("no off-diagonal blok")
    vals = symb[:5] + cbt.ravel().tolist() + bkt.ravel().tolist()
    (tmp_path / "symbname").write_text("\n".join(str(v) for v in vals) + "\n")
    monkeypatch.setenv("PASTIX_FILE_ORDER", os.path.join(d, "ordergen"))
    monkeypatch.chdir(tmp_path)
    ip, dp = px.initParam()
    ip[px.iparm.io_strategy] = int(px.io.Load)
    ip[px.iparm.ordering] = int(px.ordering.Personal)
    pd = px.init(ip, dp)
    S = spmatrix(A, mtxtype.Symmetric)
    rc = lib.pastix_task_analyze(pd.ptr, S.pointer())
    assert rc == px.error.FILE
