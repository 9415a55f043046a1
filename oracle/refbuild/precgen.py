"""Precision converter for building the reference from its sources -- TEST
INFRASTRUCTURE ONLY (it feeds ``oracle/_ref``, never the product).

PaStiX writes every numerical file once, in complex double (``z``), and its
CMake generates the real and single precision variants at build time with a
substitution engine that lives in the ``morse_cmake`` submodule.  That
submodule is not part of the reference checkout, so this module restates the
conversion: an ordered list of regex rules, each giving the text of one
construct in the four precisions (s, d, c, z); converting a ``z`` file to
precision X replaces every match of the ``z`` column by the X column.  The
PaStiX-specific rows follow ``cmake_modules/local_subs.py:18-99`` (types,
``zone``/``zzero``, the ``cpucblk_``/``core_``/``bvec_``... prefixes); the
generic rows (BLAS / LAPACKE names, the complex helpers that vanish in real
arithmetic) are written here from the BLAS naming rules.  Only the files the
oracle build needs are converted, and the rule set covers exactly them.

Mixed-precision files (``@precisions mixed zc -> ds``) use the second table.
"""
from __future__ import annotations

import re

PRECS = ("s", "d", "c", "z")

# (s, d, c, z): z is a regex, the others replacement strings.  Applied in order.
_NORMAL = [
    # --- complex helpers that disappear in real arithmetic (must run first)
    ("", "", "CBLAS_SADDR", r"\bCBLAS_SADDR"),
    ("", "", "crealf", r"\bcreal(?=\s*\()"),
    ("0.*", "0.*", "cimagf", r"\bcimag(?=\s*\()"),
    ("", "", "conjf", r"\bconj(?=\s*\()"),
    ("fabsf", "fabs", "cabsf", r"\bcabs(?=\s*\()"),
    ("sqrtf", "sqrt", "csqrtf", r"\bcsqrt(?=\s*\()"),
    ("CblasTrans", "CblasTrans", "CblasConjTrans", r"\bCblasConjTrans\b"),
    ("PastixTrans", "PastixTrans", "PastixConjTrans", r"\bPastixConjTrans\b"),
    # --- types (local_subs.py:26-31)
    ("float", "double", "pastix_complex32_t", r"\bpastix_complex64_t\b"),
    ("float", "float", "pastix_complex32_t", r"\bpastix_complex32_t\b"),
    ("float", "double", "spm_complex32_t", r"\bspm_complex64_t\b"),
    ("SpmFloat", "SpmDouble", "SpmComplex32", r"\bSpmComplex64\b"),
    ("PastixFloat", "PastixDouble", "PastixComplex32", r"\bPastixComplex64\b"),
    ("PastixFloat", "PastixFloat", "PastixComplex32", r"\bPastixComplex32\b"),
    ("PASTIX_MPI_FLOAT", "PASTIX_MPI_DOUBLE", "PASTIX_MPI_COMPLEX32", r"\bPASTIX_MPI_COMPLEX64\b"),
    # real-valued quantities of a complex file (norms, thresholds) follow the base precision
    ("float", "double", "float", r"\bdouble\b"),
    # --- BLAS / LAPACKE names whose real form differs from the plain z -> d swap
    ("cblas_snrm2", "cblas_dnrm2", "cblas_scnrm2", r"\bcblas_dznrm2\b"),
    ("cblas_sscal", "cblas_dscal", "cblas_csscal", r"\bcblas_zdscal\b"),
    ("cblas_isamax", "cblas_idamax", "cblas_icamax", r"\bcblas_izamax\b"),
    ("cblas_ssyrk", "cblas_dsyrk", "cblas_cherk", r"\bcblas_zherk\b"),
    ("cblas_ssyr", "cblas_dsyr", "cblas_cher", r"\bcblas_zher\b"),
    ("cblas_sger", "cblas_dger", "cblas_cgerc", r"\bcblas_zgerc\b"),
    ("cblas_sger", "cblas_dger", "cblas_cgeru", r"\bcblas_zgeru\b"),
    ("cblas_sdot", "cblas_ddot", "cblas_cdotc_sub", r"\bcblas_zdotc_sub\b"),
    ("cblas_sdot", "cblas_ddot", "cblas_cdotu_sub", r"\bcblas_zdotu_sub\b"),
    ("LAPACKE_slansy", "LAPACKE_dlansy", "LAPACKE_clanhe", r"\bLAPACKE_zlanhe"),
    ("LAPACKE_sormqr", "LAPACKE_dormqr", "LAPACKE_cunmqr", r"\bLAPACKE_zunmqr"),
    ("LAPACKE_sormlq", "LAPACKE_dormlq", "LAPACKE_cunmlq", r"\bLAPACKE_zunmlq"),
    ("LAPACKE_sorgqr", "LAPACKE_dorgqr", "LAPACKE_cungqr", r"\bLAPACKE_zungqr"),
    ("LAPACKE_slag2d", "LAPACKE_slag2d", "LAPACKE_clag2z", r"\bLAPACKE_clag2z"),
    ("LAPACKE_slag2d", "LAPACKE_dlag2s", "LAPACKE_clag2z", r"\bLAPACKE_zlag2c"),
    ("LAPACKE_slamch", "LAPACKE_dlamch", "LAPACKE_slamch", r"\bLAPACKE_dlamch"),
    ("LAPACKE_slassq", "LAPACKE_dlassq", "LAPACKE_classq", r"\bLAPACKE_zlassq"),
    ("slassq", "dlassq", "slassq", r"\bdlassq\b"),
    ("cblas_s", "cblas_d", "cblas_c", r"\bcblas_z"),
    ("cblas_s", "cblas_d", "cblas_s", r"\bcblas_d(?=[a-z])"),
    ("LAPACKE_s", "LAPACKE_d", "LAPACKE_c", r"\bLAPACKE_z"),
    ("LAPACKE_s", "LAPACKE_d", "LAPACKE_s", r"\bLAPACKE_d(?=[a-z])"),
    ("MYLAPACKE_s", "MYLAPACKE_d", "MYLAPACKE_c", r"\bMYLAPACKE_z"),
    # --- flop macros (common/flops.h defines all four)
    ("FLOPS_S", "FLOPS_D", "FLOPS_C", r"\bFLOPS_Z"),
    # --- PaStiX constants (local_subs.py:51-52)
    ("sone", "done", "cone", r"zone\b"),
    ("szero", "dzero", "czero", r"zzero\b"),
    # --- dot products: the conjugated and plain forms are one function in real arithmetic
    ("sdot", "ddot", "cdotc", r"(?<=_)zdotc"),
    ("sdot", "ddot", "cdotu", r"(?<=_)zdotu"),
    # --- PaStiX prefixes (local_subs.py:55-75) and the other z-marked names
    (r"\1s", r"\1d", r"\1c",
     r"\b((?:__|pthread_)?(?:cpucblk|cpublok|core|coeftab|bvec|bcsc|solve_cblk|solve_blok|solve|args|sequential"
     r"|static|dynamic|runtime|starpu|parsec|sopalin|thread|pastix|gpucblk|gpublok|gpu|cuda|csc|blok|cblk|task"
     r"|vec|spm|_pastix|_coeftab|_bcsc|_cpucblk)_)z(?=[a-z_.])"),
    (r"s_", r"d_", r"c_", r"\bz_(?=[a-zA-Z])"),
    (r"_s_", r"_d_", r"_c_", r"\b_z_(?=[a-z])"),
    (r"s\1", r"d\1", r"c\1", r"\bz(potrf|getrf|sytrf|hetrf|pxtrf|trsm|diag|gemm|spmv)(?=_)"),
    (r"s\1", r"d\1", r"c\1", r"\bz(lr[a-z0-9_]*|ge2lr[a-z0-9_]*|rradd[a-z0-9_]*|_nan_check)\b"),
]

# @precisions mixed zc -> ds
_MIXED = [
    ("double", r"\bpastix_complex64_t\b"),
    ("float", r"\bpastix_complex32_t\b"),
    ("double", r"\bspm_complex64_t\b"),
    ("LAPACKE_dlag2s", r"\bLAPACKE_zlag2c"),
    ("LAPACKE_slag2d", r"\bLAPACKE_clag2z"),
    ("coeftab_dcblk", r"\bcoeftab_zcblk"),
    ("coeftab_ds", r"\bcoeftab_zc"),
    ("cpucblk_ds", r"\bcpucblk_zc"),
    ("pastix_dscores", r"\bpastix_zccores"),
    ("pastix_dcores", r"\bpastix_zcores"),
    ("pastix_ds", r"\bpastix_zc"),
    ("pastix_scores", r"\bpastix_ccores"),
    ("cpucblk_s", r"\bcpucblk_c(?=[a-z])"),
    ("cpucblk_d", r"\bcpucblk_z(?=[a-z])"),
    ("DSOVERFCHECK", r"\bZCOVERFCHECK\b"),
    ("PastixDouble", r"\bPastixComplex64\b"),
    ("PastixFloat", r"\bPastixComplex32\b"),
]

_COMPILED = None


def _compiled():
    global _COMPILED
    if _COMPILED is None:
        normal = [(re.compile(row[3]), {p: row[i] for i, p in enumerate(PRECS[:3])}) for row in _NORMAL]
        # a mixed name may follow an underscore (include guards): no word boundary there
        mixed = [(re.compile(pat.replace(r"\b", r"(?<![A-Za-z0-9])", 1)), rep) for rep, pat in _MIXED]
        _COMPILED = (normal, mixed)
    return _COMPILED


def convert(text: str, prec: str) -> str:
    """The z (or zc) source text in precision ``prec`` (s, d, c; ds for mixed)."""
    normal, mixed = _compiled()
    if prec == "z" or prec == "zc":
        return text
    if prec == "ds":
        for rx, rep in mixed:
            text = rx.sub(rep, text)
        return text
    for rx, reps in normal:
        text = rx.sub(reps[prec], text)
    return text


def convert_name(name: str, prec: str) -> str:
    """File name of the converted file: the z marker of the name replaced."""
    if prec in ("z", "zc"):
        return name
    if prec == "ds":
        return name.replace("zc", "ds", 1)
    if name.startswith("z_"):
        return prec + name[1:]
    m = re.match(r"^(.*?)(z)(?=[a-z_.])", name)
    if m is None:
        raise ValueError(name)
    i = m.end(1)
    return name[:i] + prec + name[i + 1:]
