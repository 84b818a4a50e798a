"""The Julia glue (julia/HaissinskiGPU.jl) against the C ABI, read as text.

Julia is not installed here, so the glue cannot run; these checks keep it
in step with the header: its struct mirrors have the fields, order and widths
of the ctypes mirrors (which the ABI tests compare with the C layouts), and
every ccall, in the glue and in the integration guide's examples, names an
exported entry point with the argument count and kinds of its declaration."""
import ctypes
import os
import re

import pytest

from haissinskijulia_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GLUE = os.path.join(ROOT, "julia", "HaissinskiGPU.jl")

# Julia spellings of the reference's field names -> the C/ctypes names
_FIELD = {"α_c": "alpha_c", "ϕs": "phi_s", "update_η": "update_eta"}
_JL_SIZE = {"Float64": 8, "Int64": 8, "UInt64": 8, "Int32": 4, "UInt8": 1, "Ptr{Float64}": 8}


def _glue() -> str:
    with open(GLUE, encoding="utf-8") as f:
        return f.read()


def _jl_structs(src: str) -> dict:
    out = {}
    for m in re.finditer(r"^struct (\w+)\n(.*?)^end", src, re.S | re.M):
        fields = re.findall(r"^\s+(\S+)::(\S+)\s*$", m.group(2), re.M)
        out[m.group(1)] = fields
    return out


def _ctypes_fields(cls) -> list:
    out = []
    for name, typ in cls._fields_:
        if issubclass(typ, ctypes.Array):          # padding bytes
            out += [(f"{name}{i}", ctypes.sizeof(typ._type_)) for i in range(typ._length_)]
        else:
            out.append((name, ctypes.sizeof(typ)))
    return out


@pytest.mark.parametrize("name", ["HjParams", "HjWake", "HjGrid", "HjResult"])
def test_struct_mirrors_match_the_ctypes_layouts(name):
    jl = _jl_structs(_glue())[name]
    ct = _ctypes_fields(getattr(_lib, name))
    assert len(jl) == len(ct), name
    for (jn, jt), (cn, cs) in zip(jl, ct):
        assert _JL_SIZE[jt] == cs, f"{name}.{jn}: {jt} vs {cs} bytes"
        if not cn.startswith("_pad"):
            assert _FIELD.get(jn, jn) == cn, f"{name}: {jn} vs {cn}"


def _kind_jl(t: str) -> str:
    t = t.strip()
    if t.startswith(("Ptr", "Ref", "Cstring")):
        return "ptr"
    return {"Int32": "i32", "Int64": "i64", "UInt64": "u64", "Float64": "f64",
            "Cvoid": "void"}[t]


def _kind_ct(t) -> str:
    if t is None:
        return "void"
    if t in (ctypes.c_void_p, ctypes.c_char_p) or hasattr(t, "_type_") and \
            isinstance(t._type_, type):
        return "ptr"
    return {ctypes.c_int32: "i32", ctypes.c_int64: "i64", ctypes.c_uint64: "u64",
            ctypes.c_double: "f64"}[t]


def _split_types(s: str) -> list:
    """Top-level comma split of a Julia type tuple body."""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "{(":
            depth += 1
        elif ch in "})":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur)
    return [t.strip() for t in out if t.strip()]


_CCALL = r"ccall\(\(:(\w+), libhj\),\s*(\w+),\s*\(((?:[^()]|\([^()]*\))*)\)"


def test_every_ccall_matches_its_declaration():
    src = _glue()
    need = {"hj_create", "hj_destroy", "hj_evolve", "hj_wake_reference", "hj_last_error",
            "hj_status_string", "hj_batch_create", "hj_batch_add_gaussian", "hj_batch_advance",
            "hj_batch_poll", "hj_batch_take_many", "hj_batch_destroy"}
    calls = re.findall(_CCALL, src, re.S)
    assert {c[0] for c in calls} >= need
    lib = _lib.SIGNATURES
    for name, ret, args in calls:
        assert name in lib, name
        res, argtypes = lib[name]
        jl_args = [_kind_jl(t) for t in _split_types(args)]
        assert jl_args == [_kind_ct(t) for t in argtypes], name
        assert _kind_jl(ret) == _kind_ct(res), name
