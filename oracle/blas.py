"""Locate a CBLAS/LAPACKE shared library for the oracle -- TEST INFRASTRUCTURE.

The oracle links no BLAS at build time.  Its CPU-baseline timing and the
reference build under ``oracle/_ref`` need an OpenBLAS that exports the plain
``cblas_*`` / ``LAPACKE_*`` names.  Search order: ``$ORACLE_BLAS``, then any
``libopenblas*.so*`` shipped inside a wheel of the running interpreter's
site-packages (wheels vendor their native libraries next to the package, in
``<pkg>.libs/`` or ``<pkg>/``).  Libraries with a symbol prefix (SciPy's
``libscipy_openblas``) are skipped: their names do not match CBLAS.
"""
from __future__ import annotations

import glob
import os
import site
import sys
from pathlib import Path


def candidates() -> list[Path]:
    out = []
    env = os.environ.get("ORACLE_BLAS", "")
    if env:
        out.append(Path(env))
    roots = []
    try:
        roots += site.getsitepackages()
    except AttributeError:
        pass
    roots.append(os.path.join(sys.prefix, "lib"))
    seen = set()
    for r in roots:
        for pat in ("*.libs/libopenblas*.so*", "*/libopenblas*.so*"):
            for p in sorted(glob.glob(os.path.join(r, pat))):
                if "scipy_openblas" in p or p in seen:
                    continue
                seen.add(p)
                out.append(Path(p))
    return [p for p in out if p.exists()]


def find_openblas() -> Path | None:
    c = candidates()
    return c[0] if c else None


def runtime_deps(lib: Path) -> list[Path]:
    """The wheel's bundled gfortran / quadmath that the OpenBLAS needs loaded first."""
    d = lib.parent
    return sorted(d.glob("libquadmath*.so*")) + sorted(d.glob("libgfortran*.so*"))
