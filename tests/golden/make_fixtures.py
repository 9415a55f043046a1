"""Converts the reference's own test matrices into compact npz fixtures.

Reads test/matrix/orsirr.rua (real unsymmetric, n=1030; the reference's LU
test, example/CTestLists.txt:121,148-149) and test/matrix/small.rsa (real
symmetric indefinite KKT, n=12111; the LDL^T test with
dparm_epsilon_magn_ctrl 1e-14, example/CTestLists.txt:117,147) in the
Harwell-Boeing format and writes tests/golden/{orsirr,small}.npz with the CSC
arrays (0-based).  Run once where the reference tree is available:
    python tests/golden/make_fixtures.py /path/to/pastix
"""
from __future__ import annotations

import re
import sys
from pathlib import Path

import numpy as np


def _fields(lines, fmt, count, conv):
    m = re.match(r"\((\d*)(?:1P)?\s*(\d*)([IiEeDdFf])(\d+)", fmt.replace(" ", ""))
    if m is None:
        raise ValueError(fmt)
    per = int(m.group(2) or m.group(1) or 1) if m.group(2) else int(m.group(1) or 1)
    width = int(m.group(4))
    out = []
    for ln in lines:
        ln = ln.rstrip("\n")
        for i in range(per):
            s = ln[i * width:(i + 1) * width].strip()
            if s:
                out.append(conv(s.replace("D", "E").replace("d", "e")))
        if len(out) >= count:
            break
    return out[:count]


def read_hb(path: Path):
    with open(path) as f:
        lines = f.readlines()
    ptrcrd, indcrd, valcrd, rhscrd = (int(x) for x in lines[1].split()[1:5])
    mxtype = lines[2][:3].upper()
    nrow, ncol, nnz = (int(x) for x in lines[2][3:].split()[:3])
    fmts = re.findall(r"\([^)]*\)", lines[3])
    start = 5 if rhscrd > 0 else 4
    p = lines[start:start + ptrcrd]
    i = lines[start + ptrcrd:start + ptrcrd + indcrd]
    v = lines[start + ptrcrd + indcrd:start + ptrcrd + indcrd + valcrd]
    colptr = np.array(_fields(p, fmts[0], ncol + 1, int), dtype=np.int64) - 1
    rowind = np.array(_fields(i, fmts[1], nnz, int), dtype=np.int64) - 1
    values = np.array(_fields(v, fmts[2], nnz, float), dtype=np.float64)
    return mxtype, nrow, colptr, rowind, values


def main(ref: Path):
    out = Path(__file__).resolve().parent
    for name, fn in (("orsirr", "orsirr.rua"), ("small", "small.rsa")):
        mxtype, n, cp, ri, va = read_hb(ref / "test" / "matrix" / fn)
        np.savez_compressed(out / f"{name}.npz", mxtype=mxtype, n=n, colptr=cp.astype(np.int32),
                            rowind=ri.astype(np.int32), values=va)
        print(name, mxtype, n, va.size)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_fixtures.py <path of the PaStiX source tree>")
    main(Path(sys.argv[1]))
