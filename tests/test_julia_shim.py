"""The Julia shim (juliatdgl_b200/julia/TDGLB200.jl) against the C-ABI: no Julia is installed here, so its structs
are read as text and checked field by field, in order and by type, against the Python mirror (juliatdgl_b200/abi.py,
whose layout the C-ABI tests pin to include/tdgl_b200.h), and every C function it calls must be one the header
declares and the library exports."""
import ctypes as C
import os
import re

import pytest

from juliatdgl_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "juliatdgl_b200", "julia", "TDGLB200.jl")
HEADER = os.path.join(ROOT, "include", "tdgl_b200.h")


def julia_structs(text):
    """{name: [(field, type)]} of the `struct` / `mutable struct` blocks whose fields are one per line."""
    out = {}
    for m in re.finditer(r"^(?:mutable )?struct (\w+)\n(.*?)^end", text, re.S | re.M):
        fields = []
        for line in m.group(2).splitlines():
            line = line.split("#")[0].strip()
            for part in line.split(";"):
                part = part.strip()
                if "::" in part:
                    n, t = part.split("::", 1)
                    fields.append((n.strip(), t.strip()))
        out[m.group(1)] = fields
    return out


CONST = {"MAXB": abi.MAXB, "MAXSTG": 64, "MAXMAT": 8}


def julia_to_ctypes_size(t):
    """Byte size and element count of a Julia field type, with the struct types resolved from abi."""
    t = t.strip()
    m = re.fullmatch(r"NTuple\{(\w+),(.*)\}", t)
    if m:
        n = int(CONST.get(m.group(1), m.group(1)) if not m.group(1).isdigit() else m.group(1))
        return n * julia_to_ctypes_size(m.group(2))
    scal = {"Int32": 4, "UInt64": 8, "Int64": 8, "Float64": 8, "UInt8": 1}
    if t in scal:
        return scal[t]
    if t.startswith("Ptr{"):
        return 8
    structs = {"Grid_t": abi.Grid_t, "BandCoef_t": abi.BandCoef_t}
    return C.sizeof(structs[t])


@pytest.mark.parametrize("jl,py", [("Grid_t", abi.Grid_t), ("BandCoef_t", abi.BandCoef_t),
                                   ("Materials_t", abi.Materials_t), ("Params_t", abi.Params_t),
                                   ("StateView_t", abi.StateView_t), ("CarryView_t", abi.CarryView_t)])
def test_shim_structs_match_the_abi(jl, py):
    structs = julia_structs(open(SHIM).read())
    assert jl in structs, jl
    jf = structs[jl]
    pf = py._fields_
    assert [n for n, _ in jf] == [n for n, _ in pf], jl
    for (n, t), (pn, pt) in zip(jf, pf):
        assert julia_to_ctypes_size(t) == C.sizeof(pt), (jl, n, t)
    # the whole struct, padding included, has the C size (Julia lays structs out as C does)
    total = 0
    for n, t in jf:
        sz = julia_to_ctypes_size(t)
        al = min(8, sz) if sz in (1, 2, 4, 8) else 8
        total = (total + al - 1) // al * al + sz
    assert (total + 7) // 8 * 8 == C.sizeof(py), jl


def test_shim_calls_declared_entry_points():
    text = open(SHIM).read()
    called = set(re.findall(r"ccall\(\(:(\w+), LIB\)", text))
    header = open(HEADER).read()
    declared = set(re.findall(r"\b(tdgl_\w+)\s*\(", header))
    assert called and called <= declared, called - declared
    assert {"tdgl_ctx_create", "tdgl_upload_state", "tdgl_set_carry", "tdgl_steps", "tdgl_download_state",
            "tdgl_get_carry", "tdgl_supported", "tdgl_abi_version"} <= called


def test_shim_abi_version_is_the_headers():
    text = open(SHIM).read()
    v = int(re.search(r"const ABI_VERSION = Int32\((\d+)\)", text).group(1))
    h = int(re.search(r"#define TDGL_ABI_VERSION (\d+)", open(HEADER).read()).group(1))
    assert v == h == abi.ABI_VERSION
