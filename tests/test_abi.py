"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: this runs without a GPU)."""
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(ddm_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_builds_and_exports_all_declared_symbols():
    from hackathon_b200 import build
    lib = build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True, check=True)
    exported = set(re.findall(r"\bT (ddm_[a-z0-9_]+)", out.stdout))
    declared = _declared()
    assert declared, "no declarations found"
    assert declared <= exported, f"missing: {sorted(declared - exported)}"


def test_ctypes_signatures_cover_header():
    from hackathon_b200 import _lib
    assert _declared() <= set(_lib.exported_symbols())
    _lib.load()  # resolves every symbol


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import hackathon_b200 as H
    with pytest.raises(H.DdmError) as e:
        H.DdmEngine.create()
    assert e.value.code == 5  # DDM_ERR_NODEV


def test_invalid_geometry_rejected_before_device():
    import hackathon_b200 as H
    for kw in (dict(N=100), dict(N=64, T=64, L=65), dict(N=64, T=64, TPAD=100),
               dict(N=64, NB=0), dict(N=64, knodes=0)):
        with pytest.raises(H.DdmArgError):
            H.DdmEngine.create(**kw)
