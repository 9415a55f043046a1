"""Recipe: compile the reference PaStiX from its own sources into
``oracle/_ref/libpastix_ref.so`` -- TEST INFRASTRUCTURE ONLY.

The reference's CMake cannot run here (the ``spm`` and ``morse_cmake``
submodules are absent), so this script does what it would do for a
one-process, CPU-only build:

* generates the real / single precision sources and headers from the ``z``
  files with ``precgen`` (the reference's precision generator is part of the
  missing submodule), into ``oracle/_ref/gen``;
* compiles the analysis (graph, order, symbol, blend), the numerical phase
  (bcsc, sopalin, kernels, refinement) and the common layer as listed in the
  reference's ``CMakeLists.txt:573-833`` and ``kernels/CMakeLists.txt``,
  without MPI, hwloc, StarPU, PaRSEC, CUDA, Scotch or Metis, against the
  restated SpM shim (``shim/``), with ``-DPASTIX_INT64``;
* compiles ``ref_driver.c`` (this repository's C entry points for the tests);
* links everything with an OpenBLAS found by ``oracle/blas.py``.  Functions
  that nothing built defines (complex single precision, the low-rank
  kernels) become stubs that abort, so the library loads; the oracle never
  calls them.  Their names are listed in ``oracle/_ref/stubbed.txt``.

Nothing from the reference is copied into the repository: sources are read
where they lie and every output goes to ``oracle/_ref``.

Usage: python oracle/refbuild/build_ref.py [path of the PaStiX source tree]
(default: $PASTIX_SOURCE_DIR, else /root/reference).
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parent.parent))
import precgen  # noqa: E402

OUT = HERE.parent / "_ref"
GEN = OUT / "gen"
OBJ = OUT / "obj"
LIB = OUT / "libpastix_ref.so"

PLAIN = """
graph/graph.c graph/graph_compute_projection.c graph/graph_connected_components.c graph/graph_io.c
graph/graph_isolate.c graph/graph_prepare.c
order/order.c order/order_add_isolate.c order/order_amalgamate.c order/order_apply_level_order.c
order/order_check.c order/order_compute_personal.c order/order_find_supernodes.c order/order_grids.c
order/order_io.c order/pastix_subtask_order.c
symbol/fax_csr.c symbol/fax_csr_amalgamate.c symbol/fax_csr_direct.c symbol/fax_csr_iluk.c symbol/symbol.c
symbol/symbol_base.c symbol/symbol_check.c symbol/symbol_cost.c symbol/symbol_cost_flops.c
symbol/symbol_cost_perfs.c symbol/symbol_draw.c symbol/symbol_draw_map.c symbol/symbol_expand.c
symbol/symbol_fax_direct.c symbol/symbol_fax_iluk.c symbol/symbol_io.c symbol/symbol_reorder.c
symbol/symbol_reordering.c symbol/pastix_subtask_reordering.c symbol/pastix_subtask_symbfact.c
blend/pastix_subtask_blend.c blend/pastix_task_analyze.c blend/blendctrl.c blend/cand.c blend/cand_gendot.c
blend/cost.c blend/elimintree.c blend/extendVector.c blend/extracblk.c blend/propmap.c blend/simu.c
blend/simu_run.c blend/simu_task.c blend/solver.c blend/solver_backup.c blend/solver_check.c
blend/solver_copy.c blend/solver_draw.c blend/solver_io.c blend/solver_matrix_gen.c
blend/solver_matrix_gen_utils.c blend/solver_recv.c blend/splitsymbol.c
common/api.c common/integer.c common/isched.c common/models.c common/get_options.c common/parse_options.c
common/check_options.c common/getline.c common/isched_nohwloc.c
bcsc/bcsc.c bcsc/bvec.c
sopalin/coeftab.c sopalin/schur.c sopalin/diag.c sopalin/pastix_task_sopalin.c sopalin/pastix_task_solve.c
sopalin/pastix.c sopalin/pastix_rhs.c
refinement/pastix_task_refine.c
kernels/kernels.c kernels/kernels_trace.c kernels/lowrank.c kernels/queue.c
""".split()

# z headers generated in every precision the includers name
HEADERS = {
    "bcsc/bcsc_z.h": "sdcz",
    "sopalin/coeftab_z.h": "sdcz",
    "refinement/z_refine_functions.h": "sdcz",
    "kernels/pastix_zcores.h": "sdcz",
    "kernels/pastix_zcuda.h": "sdcz",
    "kernels/pastix_zlrcores.h": "sdcz",
    "kernels/z_nan_check.h": "sdcz",
    "kernels/cpucblk_zpack.h": "sdcz",
}
MIXED_HEADERS = ["kernels/pastix_zccores.h"]

# z sources compiled in double, single and complex double (complex single is stubbed)
SOURCES = """
common/z_integer.c
bcsc/bcsc_zinit.c bcsc/bcsc_znorm.c bcsc/bcsc_zspmv.c bcsc/bvec_zcompute.c bcsc/bvec_zlapmr.c bcsc/bvec_zmpi_comm.c
sopalin/coeftab_z.c sopalin/coeftab_zinit.c sopalin/sequential_zdiag.c sopalin/sequential_zgetrf.c
sopalin/sequential_zpotrf.c sopalin/sequential_zsytrf.c sopalin/sequential_ztrsm.c
refinement/z_refine_bicgstab.c refinement/z_refine_functions.c refinement/z_refine_gmres.c
refinement/z_refine_grad.c refinement/z_refine_pivot.c
kernels/core_zgemdm.c kernels/core_zgetmo.c kernels/core_zgeadd.c kernels/core_zplrnt.c kernels/core_ztradd.c
kernels/core_zgemmsp.c kernels/core_ztrsmsp.c kernels/core_zscalo.c kernels/core_zsytrfsp.c
kernels/core_zpotrfsp.c kernels/core_zgetrfsp.c
kernels/cpucblk_zinit.c kernels/cpucblk_zdiff.c kernels/cpucblk_zadd.c kernels/cpucblk_zschur.c
kernels/cpublok_zadd.c kernels/cpucblk_zmpi_coeftab.c kernels/cpucblk_zmpi_rhs_fwd.c
kernels/cpucblk_zmpi_rhs_bwd.c kernels/cpucblk_zpack.c kernels/solve_ztrsmsp.c kernels/cpucblk_zcompress.c
""".split()
# complex-only sources of the z build (the LL^H / LDL^H kernels the z dispatch tables name)
Z_ONLY = """
sopalin/sequential_zhetrf.c sopalin/sequential_zpxtrf.c kernels/core_zhetrfsp.c kernels/core_zpxtrfsp.c
""".split()
MIXED_SOURCES = ["sopalin/coeftab_zcinit.c", "kernels/cpucblk_zcinit.c"]

SOURCE_PRECS = "sdz"


def ref_root(argv=()) -> Path:
    if len(argv) > 1:
        return Path(argv[1])
    return Path(os.environ.get("PASTIX_SOURCE_DIR", "/root/reference"))


def _write(path: Path, text: str) -> None:
    path.parent.mkdir(parents=True, exist_ok=True)
    if path.exists() and path.read_text() == text:
        return  # keep the timestamp: no rebuild of unchanged files
    path.write_text(text)


def generate(src: Path) -> list[tuple[Path, str]]:
    """Writes the converted headers and sources; returns (source, precision) pairs to compile."""
    for rel, precs in HEADERS.items():
        text = (src / rel).read_text()
        d = Path(rel).parent
        for p in precs:
            _write(GEN / d / precgen.convert_name(Path(rel).name, p), precgen.convert(text, p))
    for rel in MIXED_HEADERS:
        d = Path(rel).parent
        _write(GEN / d / precgen.convert_name(Path(rel).name, "ds"), precgen.convert((src / rel).read_text(), "ds"))
    units = []
    for rel in SOURCES:
        text = (src / rel).read_text()
        d = Path(rel).parent
        for p in SOURCE_PRECS:
            if p == "z":
                units.append((src / rel, "z"))
                continue
            out = GEN / d / precgen.convert_name(Path(rel).name, p)
            _write(out, precgen.convert(text, p))
            units.append((out, p))
    for rel in Z_ONLY:
        units.append((src / rel, "z"))
    for rel in MIXED_SOURCES:
        d = Path(rel).parent
        out = GEN / d / precgen.convert_name(Path(rel).name, "ds")
        _write(out, precgen.convert((src / rel).read_text(), "ds"))
        units.append((out, "ds"))
        units.append((src / rel, "zc"))
    for rel in PLAIN:
        units.append((src / rel, ""))
    return units


def include_flags(src: Path) -> list[str]:
    dirs = [HERE / "shim", GEN, GEN / "kernels", GEN / "bcsc", GEN / "sopalin", GEN / "refinement",
            src, src / "include", src / "common", src / "kernels", src / "bcsc", src / "sopalin", src / "refinement"]
    return [f"-I{d}" for d in dirs]


# -DNDEBUG as in an optimized build: one debug assertion of the reference
# (blend/solver_matrix_gen_utils.c:514-515) compares the rows of a symbol blok,
# counted in nodes, with those of its solver blok, counted in unknowns, and so
# fails for dof > 1 matrices whose supernodes are wide enough for 2D tasks.
CFLAGS = ["-O2", "-g0", "-fPIC", "-std=gnu11", "-w", "-Drestrict=", "-pthread", "-fno-strict-aliasing", "-DNDEBUG"]
# the comparison helper of ref_driver.c runs its loop with OpenMP
DRIVER_FLAGS = ["-fopenmp"]


def _obj_name(path: Path, prec: str, src: Path) -> Path:
    try:
        rel = path.relative_to(src)
        tag = "ref"
    except ValueError:
        if GEN in path.parents:
            rel, tag = path.relative_to(GEN), "gen"
        else:
            rel, tag = Path(path.name), "own"
    return OBJ / tag / (prec or "x") / rel.with_suffix(".o")


def compile_unit(path: Path, prec: str, src: Path) -> tuple[Path, str | None]:
    obj = _obj_name(path, prec, src)
    if obj.exists() and obj.stat().st_mtime >= path.stat().st_mtime:
        return obj, None
    obj.parent.mkdir(parents=True, exist_ok=True)
    flags = list(CFLAGS)
    if path.name == "ref_driver.c":
        flags += DRIVER_FLAGS
    if prec:
        flags.append(f"-DPRECISION_{prec}")
    cmd = ["gcc", *flags, *include_flags(src), "-c", str(path), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{path} [{prec}]\n{r.stderr[-4000:]}"
    return obj, None


def _undefined(log: str) -> list[str]:
    return sorted(set(re.findall(r"undefined reference to `([^'`]+)'", log)))


def link(objs: list[Path], blas: Path) -> None:
    base = ["gcc", "-shared", "-o", str(LIB), *map(str, objs), str(blas), f"-Wl,-rpath,{blas.parent}",
            "-lm", "-lpthread", "-fopenmp", "-Wl,--no-undefined"]
    r = subprocess.run(base, capture_output=True, text=True)
    if r.returncode == 0:
        (OUT / "stubbed.txt").write_text("")
        return
    missing = _undefined(r.stderr)
    if not missing:
        raise RuntimeError(r.stderr[-4000:])
    stub = OUT / "stubs.c"
    lines = ["#include <stdio.h>", "#include <stdlib.h>",
             "static void oracle_stub(const char *n) { fprintf(stderr, \"oracle build: %s is not built\\n\", n); abort(); }"]
    lines += [f"void {m}(void) {{ oracle_stub(\"{m}\"); }}" for m in missing]
    _write(stub, "\n".join(lines) + "\n")
    sobj = OBJ / "stubs.o"
    subprocess.run(["gcc", "-fPIC", "-w", "-c", str(stub), "-o", str(sobj)], check=True)
    r = subprocess.run(base[:5] + [str(sobj)] + base[5:], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stderr[-4000:])
    (OUT / "stubbed.txt").write_text("\n".join(missing) + "\n")


def build(src: Path | None = None, jobs: int | None = None) -> Path:
    src = src or ref_root()
    if not (src / "sopalin" / "pastix_task_sopalin.c").exists():
        raise FileNotFoundError(f"no PaStiX source tree at {src}")
    from oracle import blas as blasmod
    blas = blasmod.find_openblas()
    if blas is None:
        raise FileNotFoundError("no OpenBLAS with CBLAS/LAPACKE names found")
    OUT.mkdir(parents=True, exist_ok=True)
    stamp = OUT / "cflags.txt"
    if not stamp.exists() or stamp.read_text() != " ".join(CFLAGS):
        import shutil
        shutil.rmtree(OBJ, ignore_errors=True)  # objects of other flags
        if LIB.exists():
            LIB.unlink()
        stamp.write_text(" ".join(CFLAGS))
    units = generate(src)
    for own in ("shim/spm_min.c", "shim/missing.c", "ref_driver.c"):
        units.append((HERE / own, ""))
    errors, objs = [], []
    with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for obj, err in ex.map(lambda u: compile_unit(u[0], u[1], src), units):
            objs.append(obj)
            if err:
                errors.append(err)
    if errors:
        raise RuntimeError(f"{len(errors)} compile errors\n" + "\n".join(errors[:6]))
    newest = max(o.stat().st_mtime for o in objs)
    if not LIB.exists() or LIB.stat().st_mtime < newest:
        link(objs, blas)
    return LIB


if __name__ == "__main__":
    print(build(ref_root(sys.argv)))
