"""CPU checks of the C ABI: the library loads, exports every entry point the
header declares, keeps the reference's parameter indices, and its numerical
entry points fail loudly without a GPU (no CPU fallback)."""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, gpu_available

HEADER = ROOT / "include" / "pastix_b200.h"


def declared_functions():
    src = HEADER.read_text()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:void|int)\s*\*?\s*([A-Za-z_]\w*)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_matches_header(lib):
    from pastix_b200 import _lib
    assert sorted(_lib.EXPORTS) == declared_functions()


def _enum_names(name):
    src = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    m = re.search(r"typedef enum %s \{(.*?)\}" % name, src, re.S)
    return [x.strip() for x in m.group(1).split(",") if x.strip()]


def test_parameter_indices():
    from pastix_b200 import pastix as px
    ip = _enum_names("pastix_iparm_e")
    dp = _enum_names("pastix_dparm_e")
    assert ip[-1] == "IPARM_SIZE" and len(ip) - 1 == int(px.iparm.size)
    assert dp[-1] == "DPARM_SIZE" and len(dp) - 1 == int(px.dparm.size)
    for e in px.iparm:
        if e.name in ("size", "float_"):
            continue
        assert ip.index("IPARM_" + e.name.upper()) == int(e), e
    for e in px.dparm:
        if e.name == "size":
            continue
        assert dp.index("DPARM_" + e.name.upper()) == int(e), e


def test_init_param_defaults(lib):
    from pastix_b200 import pastix as px
    ip, dp = px.initParam()
    # common/api.c:420-571 defaults
    assert ip[px.iparm.factorization] == px.factotype.LU
    assert ip[px.iparm.min_blocksize] == 160 and ip[px.iparm.max_blocksize] == 320
    assert ip[px.iparm.refinement] == px.refine.GMRES
    assert ip[px.iparm.itermax] == 250 and ip[px.iparm.gmres_im] == 25
    assert ip[px.iparm.mixed] == 0
    assert dp[px.dparm.epsilon_refinement] == -1.0 and dp[px.dparm.epsilon_magn_ctrl] == 0.0


def test_step_order_errors(lib):
    from pastix_b200 import gen
    from pastix_b200 import pastix as px
    from pastix_b200.spm import mtxtype, spmatrix
    ip, dp = px.initParam()
    pd = px.init(ip, dp)
    S = spmatrix(gen.laplacian7(4, 4, 4), mtxtype.Symmetric)
    with pytest.raises(px.PastixError) as e:
        px.subtask_symbfact(pd)  # before ordering
    assert e.value.code == px.error.BADPARAMETER
    with pytest.raises(px.PastixError):
        px.task_numfact(pd, S)  # before analysis
    x = np.zeros(64)
    with pytest.raises(px.PastixError):
        px.task_solve(pd, S, x)  # before numfact


def test_bad_spm_rejected(lib):
    from pastix_b200 import pastix as px
    from pastix_b200.spm import spmatrix
    import scipy.sparse as sps
    ip, dp = px.initParam()
    pd = px.init(ip, dp)
    S = spmatrix(sps.identity(5, format="csc"))
    S.spm.fmttype = 1  # CSR is not accepted
    with pytest.raises(px.PastixError):
        px.task_analyze(pd, S)


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU behaviour")
def test_numeric_without_gpu_fails_loudly(lib):
    from pastix_b200 import gen
    from pastix_b200 import pastix as px
    from pastix_b200.spm import mtxtype, spmatrix
    ip, dp = px.initParam()
    ip[px.iparm.factorization] = px.factotype.POTRF
    pd = px.init(ip, dp)
    S = spmatrix(gen.laplacian7(6, 6, 6), mtxtype.Symmetric)
    px.analyze_grid(pd, S, 6, 6, 6)
    with pytest.raises(px.PastixError) as e:
        px.task_numfact(pd, S)
    assert e.value.code == px.error.INTERNAL


def test_tuning_rejects_bad_values(lib):
    """pgpu_set_tuning checks its bucket boundaries (host only, no GPU needed)."""
    from conftest import analyse
    from pastix_b200 import gen
    from pastix_b200 import pastix as px
    pd, S, info = analyse(gen.laplacian7(8, 8, 8), (8, 8, 8), "POTRF")
    assert px.get_tuning(pd) == (32, 32, 32)
    assert lib.pgpu_set_tuning(pd.ptr, 0, 32, 32) == px.error.BADPARAMETER
    assert lib.pgpu_set_tuning(pd.ptr, 32, 32, 16) == px.error.BADPARAMETER
    assert px.get_tuning(pd) == (32, 32, 32)
    px.set_tuning(pd, 16, 16, 48)  # rebuilds the launch lists on the host
    assert px.get_tuning(pd) == (16, 16, 48)


def _enum_values(text, name):
    """{member: value} of `typedef enum <name> {...}`, implicit values counted."""
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    m = re.search(r"typedef enum %s \{(.*?)\}" % name, text, re.S)
    if m is None:
        return None
    out, nxt = {}, 0
    for item in m.group(1).split(","):
        item = item.strip()
        if not item:
            continue
        if "=" in item:
            k, v = (x.strip() for x in item.split("=", 1))
            nxt = int(v, 0) if re.fullmatch(r"-?(0x)?[0-9a-fA-F]+", v) else out[v]
        else:
            k = item
        out[k] = nxt
        nxt += 1
    return out


# the reference source tree, where this machine has one
REF_API = Path(os.environ.get("PASTIX_SOURCE_DIR", "/root/reference")) / "include" / "pastix" / "api.h"


@pytest.mark.skipif(not REF_API.exists(), reason="the reference source tree is not on this machine")
def test_enums_match_the_reference_header():
    """Every enumeration this header restates has the reference's members and
    values (include/pastix/api.h); iparm / dparm are indices into the users'
    arrays, so a shifted member would silently change a parameter."""
    ours = HEADER.read_text()
    ref = REF_API.read_text()
    names = re.findall(r"typedef enum (pastix_\w+_e)", re.sub(r"/\*.*?\*/", "", ours, flags=re.S))
    assert "pastix_iparm_e" in names and "pastix_dparm_e" in names
    for name in names:
        r = _enum_values(ref, name)
        assert r is not None, name
        o = _enum_values(ours, name)
        assert o == {k: v for k, v in r.items() if k in o}, name
        if name in ("pastix_iparm_e", "pastix_dparm_e", "pastix_error_e"):
            assert o == r, name
