"""The C ABI library loads and exports every entry point include/fmmb.h declares (CPU)."""
import os
import re
import subprocess

import numpy as np
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
    assert C.sizeof(fmmb._MethodDesc) == 56 and C.sizeof(fmmb._TreeOpts) == 48


def test_struct_layouts_match_the_header(fmmb, tmp_path):
    """Every ctypes mirror of a header struct has the C compiler's size and field offsets."""
    import ctypes as C
    mirrors = {"fmmb_method_desc": fmmb._MethodDesc, "fmmb_tree_opts": fmmb._TreeOpts,
               "fmmb_server_opts": fmmb._ServerOpts, "fmmb_request": fmmb._Request,
               "fmmb_request_info": fmmb._RequestInfo, "fmmb_stokes_densities": fmmb._StokesDensities}
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "fmmb.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'  printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l}
    for cname, py in mirrors.items():
        assert got[(cname, "size")] == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def _julia_struct_offsets(src, name):
    """Field names and C offsets of a Julia `struct` mirror of a header struct (Julia lays an
    isbits struct out as C does), read from the shim's text."""
    m = re.search(r"^struct " + name + r"\b(.*?)\bend\b", src, re.S | re.M)
    assert m, name
    sizes = {"Int32": 4, "Int64": 8, "Float64": 8, "NTuple{3,Float64}": 24}
    fields, off = [], 0
    for fname, ftype in re.findall(r"(\w+)::([\w{},]+)", m.group(1)):
        size = 8 if ftype.startswith("Ptr") else sizes[ftype]
        align = min(size, 8)
        off = (off + align - 1) // align * align
        fields.append((fname, off))
        off += size
    return fields


def test_julia_struct_layouts_match_the_mirrors(fmmb):
    """The Julia shim's structs have the fields and offsets of the ctypes mirrors (themselves
    checked against the header above), so a struct the library fills or reads from Julia has the
    header's layout."""
    src = open(os.path.join(ROOT, "flexiblefmm.jl_b200", "julia", "FlexibleFMMB200.jl")).read()
    pairs = {"MethodDesc": fmmb._MethodDesc, "TreeOpts": fmmb._TreeOpts, "ServerOpts": fmmb._ServerOpts,
             "Request": fmmb._Request, "RequestInfo": fmmb._RequestInfo, "StokesDensitiesC": fmmb._StokesDensities}
    for jname, py in pairs.items():
        got = _julia_struct_offsets(src, jname)
        want = [(f, getattr(py, f).offset) for f, _ in py._fields_]
        assert got == want, jname


def test_stokes_density_checks(fmmb):
    """stokes_densities (src/stokes_api.jl:72-83) rejects a stresslet without its stressvecs, no
    density at all, and arrays of the wrong length, before any device work."""
    n = 10
    with pytest.raises(fmmb.ArgumentError):
        fmmb.stokes_densities(n, stresslets=np.ones((n, 3)))
    with pytest.raises(fmmb.ArgumentError):
        fmmb.stokes_densities(n, stressvecs=np.ones((n, 3)))
    with pytest.raises(fmmb.ArgumentError):
        fmmb.stokes_densities(n, weights=np.ones(n))
    with pytest.raises(fmmb.DimensionMismatch):
        fmmb.stokes_densities(n, doublets=np.ones((n - 1, 3)))
    with pytest.raises(fmmb.DimensionMismatch):
        fmmb.stokes_densities(n, stokeslets=np.ones((n, 3)), weights=np.ones(n + 1))
    a = fmmb.stokes_densities(n, stokeslets=np.ones((n, 3)), doublets=np.zeros((n, 3)))
    assert a[0].shape == (n, 3) and a[1] is None and a[2] is None and a[3].shape == (n, 3) and a[4] is None


def test_square_bbox_contains_the_points(fmmb):
    """square_bbox (src/tree/tree.jl:97-113): the largest extent about the midpoint, every point
    inside; a single point gets width 1; non-finite points are an ArgumentError."""
    rng = np.random.default_rng(3)
    x = rng.standard_normal((1000, 3)) * [1.0, 3.0, 0.5] + 7.0
    o, w = fmmb.square_bbox(x)
    assert np.all(np.array(o) <= x.min(0)) and np.all(np.array(o) + w >= x.max(0))
    assert abs(w - float((x.max(0) - x.min(0)).max())) <= 1e-12 * w
    o1, w1 = fmmb.square_bbox(np.full((1, 3), 2.0))
    assert w1 == 1.0 and o1 == (1.5, 1.5, 1.5)
    bad = x.copy()
    bad[5, 2] = np.inf
    with pytest.raises(fmmb.ArgumentError):
        fmmb.square_bbox(bad)
