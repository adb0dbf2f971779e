"""The C ABI library loads and exports every entry point include/fmmb.h declares (CPU)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    src = open(os.path.join(ROOT, "include", "fmmb.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fmmb_[a-z_0-9]+)\s*\(", src)))


def test_header_lists_the_entry_points():
    names = declared()
    assert "fmmb_plan_create" in names and "fmmb_matvec" in names and len(names) >= 25


def test_library_exports_every_declared_symbol(fmmb):
    out = subprocess.run(["nm", "-D", "--defined-only", fmmb.library_path()], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (fmmb_[a-z_0-9]+)", out))
    missing = [n for n in declared() if n not in exported]
    assert not missing, missing
    for n in declared():
        getattr(fmmb.lib(), n)               # resolvable through ctypes as well


def test_python_mirror_binds_every_symbol(fmmb):
    assert set(fmmb.EXPORTS) == set(declared())


def test_version_and_no_device_error(fmmb):
    assert b"sm_100a" in fmmb.lib().fmmb_version()
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(fmmb.FMMBError):
        fmmb.Context(0)


def test_julia_shim_binds_declared_symbols():
    """The ccall shim (flexiblefmm.jl_b200/julia/FlexibleFMMB200.jl) names only entry points the header declares;
    Julia is absent here, so its calls are checked against the header by text."""
    src = open(os.path.join(ROOT, "flexiblefmm.jl_b200", "julia", "FlexibleFMMB200.jl")).read()
    called = set(re.findall(r"ccall\(\(:(fmmb_[a-z_0-9]+), libfmmb\)", src))
    assert called and called <= set(declared())


def test_struct_layouts(fmmb):
    import ctypes as C
    assert C.sizeof(fmmb._MethodDesc) == 24 and C.sizeof(fmmb._TreeOpts) == 48
