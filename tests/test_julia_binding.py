"""The Julia ccall binding (Godunov2dB200.jl) against the C header and the ctypes binding.

Julia is not installed here, so the module cannot run; what can go wrong in
it silently is its struct layouts and its ccall signatures.  This test reads
the Julia source and checks, for every struct, the field names and their
order against the C header and against _native.py, and the byte size implied
by the Julia field types (C layout rules, which Julia's isbits structs
follow) against the header's sizes; and, for every ccall, that the symbol
is declared in the header with the same number of parameters, and that every
entry point of the header is bound.
"""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
JL = os.path.join(ROOT, "2d-dns-godunov-solver-_b200", "Godunov2dB200.jl")
HEADER = os.path.join(ROOT, "include", "godunov2d.h")

# Julia struct -> (C typedef, ctypes class name)
STRUCTS = {"MeshView": ("gd2d_mesh_view", "MeshView"), "BC": ("gd2d_bc", "BC"), "Params": ("gd2d_params", "Params"),
           "Launch": ("gd2d_launch", "Launch"), "Stats": ("gd2d_stats", "Stats")}
SCALAR = {"Int64": (8, C.c_int64), "Int32": (4, C.c_int32), "Float64": (8, C.c_double)}


def split_top(s, sep=","):
    """Split on `sep` outside braces and brackets."""
    out, depth, cur = [], 0, ""
    for ch in s:
        if ch in "{[(":
            depth += 1
        elif ch in "}])":
            depth -= 1
        if ch == sep and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += ch
    if cur.strip():
        out.append(cur)
    return [x.strip() for x in out if x.strip()]


def julia_structs():
    src = open(JL).read()
    out = {}
    for name, body in re.findall(r"^struct (\w+)\n(.*?)^end", src, flags=re.M | re.S):
        fields = []
        for line in body.splitlines():
            line = line.split("#")[0].strip()
            if line:
                fname, ftype = line.split("::")
                fields.append((fname.strip(), ftype.strip()))
        out[name] = fields
    return out


def header_struct_fields(typedef):
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (typedef, typedef), src, flags=re.S).group(1)
    names = []
    for stmt in body.split(";"):
        stmt = stmt.strip()
        if not stmt:
            continue
        # "const double *x_nodes, *y_nodes" -> x_nodes, y_nodes
        parts = split_top(re.sub(r"^(const\s+)?[\w ]+?\s+(?=\**\w+\s*(\[|,|$))", "", stmt))
        for p in parts:
            names.append(re.match(r"\**\s*(\w+)", p).group(1))
    return names


def jl_size_align(t, sizes):
    """(size, alignment) of a Julia field type under C layout rules."""
    if t in SCALAR:
        return SCALAR[t][0], SCALAR[t][0]
    if t.startswith("Ptr{"):
        return 8, 8
    m = re.fullmatch(r"NTuple\{(\d+),(\w+)\}", t)
    if m:
        n, inner = int(m.group(1)), m.group(2)
        s, a = jl_size_align(inner, sizes) if inner in SCALAR else sizes[inner]
        return n * s, a
    return sizes[t]


def test_struct_fields_match_header_and_ctypes(pkg):
    N = pkg._native
    js = julia_structs()
    assert set(js) == set(STRUCTS)
    sizes = {}
    for jname in ("BC", "MeshView", "Params", "Launch", "Stats"):
        cname, pyname = STRUCTS[jname]
        fields = js[jname]
        names = [f for f, _ in fields]
        assert names == header_struct_fields(cname), jname
        assert names == [f[0] for f in getattr(N, pyname)._fields_], jname
        # C layout of the Julia field types
        off, align = 0, 1
        for _, t in fields:
            s, a = jl_size_align(t, sizes)
            off = (off + a - 1) // a * a + s
            align = max(align, a)
        size = (off + align - 1) // align * align
        sizes[jname] = (size, align)
        assert size == C.sizeof(getattr(N, pyname)), (jname, size, C.sizeof(getattr(N, pyname)))
        # field types agree with ctypes (scalars, pointers, arrays)
        for (f, t), (pf, pt) in zip(fields, getattr(N, pyname)._fields_):
            if t in SCALAR:
                assert pt is SCALAR[t][1], (jname, f)
            elif t.startswith("Ptr{"):
                assert pt is C.c_void_p, (jname, f)
            else:
                assert C.sizeof(pt) == jl_size_align(t, sizes)[0], (jname, f)


def header_prototypes():
    src = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for name, args in re.findall(r"^(?:int|const char \*)\s*(gd2d_\w+)\s*\(([^)]*)\)\s*;", src, flags=re.M):
        a = args.strip()
        out[name] = 0 if a in ("", "void") else len(split_top(a))
    return out


def test_ccalls_match_header_prototypes():
    src = open(JL).read()
    calls = re.findall(r"ccall\(\(:(\w+), lib\),\s*(\w+),\s*\(([^()]*)\)", src)
    protos = header_prototypes()
    seen = set()
    for sym, ret, argtypes in calls:
        assert sym in protos, sym
        assert ret in ("Cint", "Cstring"), (sym, ret)
        assert len(split_top(argtypes)) == protos[sym], (sym, argtypes, protos[sym])
        seen.add(sym)
    assert seen == set(protos), sorted(set(protos) - seen)


@pytest.mark.parametrize("sym", ["gd2d_setup", "gd2d_propagate", "gd2d_get_state", "gd2d_update_variables_noalloc"])
def test_ccall_argument_types_spot_checks(sym):
    """Argument types of the main calls, as the header declares them."""
    src = open(JL).read()
    argtypes = dict((s, split_top(a)) for s, _, a in re.findall(r"ccall\(\(:(\w+), lib\),\s*(\w+),\s*\(([^()]*)\)", src))
    want = {"gd2d_setup": ["Ptr{Ptr{Cvoid}}", "Int32", "Ptr{MeshView}", "Ptr{Params}", "Ref{Launch}"],
            "gd2d_propagate": ["Ptr{Cvoid}", "Int32", "Ptr{Stats}"],
            "gd2d_get_state": ["Ptr{Cvoid}", "Int32", "Ptr{Float64}", "Ptr{Float64}", "Ptr{Float64}"],
            "gd2d_update_variables_noalloc": ["Ptr{Float64}", "Ptr{Float64}", "Ptr{Float64}", "Int64", "Float64",
                                              "Ptr{Float64}", "Ptr{Cvoid}"]}
    assert argtypes[sym] == want[sym]
