"""The Fortran side of the boundary (fortran/ndyn_gpu_mod.f90) against the C
header (include/ndyn_gpu.h) and the built library, without a Fortran
compiler (none is installed here or on the GPU hosts):

  * the bind(C) derived types ndg_control and ndg_thermo list the C structs'
    fields in the same order, with interoperable kinds, so their offsets
    under C layout rules equal offsetof() in a C program compiled against
    the header;
  * every bind(C) interface names a symbol the library exports, with the
    C prototype's number of arguments, a pointer wherever Fortran passes by
    reference and a plain scalar wherever it passes by value, and the
    prototype's return type;
  * the patched dynamics calls only functions the module declares.
"""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MOD = os.path.join(ROOT, "fortran", "ndyn_gpu_mod.f90")
DYN = os.path.join(ROOT, "fortran", "dynamics_gpu.f90")
HDR = os.path.join(ROOT, "include", "ndyn_gpu.h")
LIB = os.path.join(ROOT, "ndyn_omp_b200", "lib", "libndyn_gpu.so")

KIND = {"real(c_double)": (8, "double"), "integer(c_int)": (4, "int"),
        "type(c_ptr)": (8, "ptr"), "type(c_funptr)": (8, "funptr")}


def _lines(path):
    """Fortran source lines with comments removed and '&' continuations joined"""
    out, cur = [], ""
    for raw in open(path):
        ln = raw.split("!")[0].rstrip() if '"' not in raw else raw.rstrip()
        if not ln.strip():
            continue
        s = ln.strip()
        if s.startswith("&"):
            s = s[1:].strip()
        if s.endswith("&"):
            cur += s[:-1] + " "
            continue
        out.append(cur + s)
        cur = ""
    return out


def _decls(line):
    """'real(c_double), value :: a, b(3)' -> [(kind, value, name, count)]"""
    left, right = line.split("::")
    attrs = [a.strip().lower() for a in left.split(",")]
    kind = attrs[0].replace(" ", "")
    value = "value" in attrs[1:]
    out = []
    for m in re.finditer(r"(\w+)\s*(\(([^)]*)\))?", right):
        dim = m.group(3)
        n = 1 if dim is None else (-1 if dim.strip() == "*" or ":" in dim else int(dim))
        out.append((kind, value, m.group(1).lower(), n))
    return out


def fortran_types():
    types, name = {}, None
    for ln in _lines(MOD):
        m = re.match(r"type\s*,\s*bind\(C\)\s*::\s*(\w+)", ln, re.I)
        if m:
            name = m.group(1)
            types[name] = []
            continue
        if name and re.match(r"end\s+type", ln, re.I):
            name = None
            continue
        if name:
            types[name] += _decls(ln)
    return types


def fortran_interfaces():
    funcs, cur = {}, None
    for ln in _lines(MOD):
        m = re.match(r"(integer\(c_int\)|type\(c_ptr\))\s+function\s+(\w+)\s*\(([^)]*)\)\s*"
                     r"bind\(C,\s*name=\"(\w+)\"\)", ln, re.I)
        if m:
            args = [a.strip().lower() for a in m.group(3).split(",") if a.strip()]
            cur = {"ret": m.group(1).lower(), "args": args, "decl": {}, "cname": m.group(4)}
            funcs[m.group(2)] = cur
            continue
        if cur is not None and re.match(r"end\s+function", ln, re.I):
            cur = None
            continue
        if cur is not None and "::" in ln:
            for kind, value, nm, n in _decls(ln):
                cur["decl"][nm] = (kind, value, n)
    return funcs


def c_prototypes():
    text = re.sub(r"/\*.*?\*/", " ", open(HDR).read(), flags=re.S)
    protos = {}
    for m in re.finditer(r"\b(int|const char \*|long long|void)\s*(\w+)\s*\(([^;{]*?)\)\s*;", text):
        params = [p.strip() for p in m.group(3).split(",") if p.strip() and p.strip() != "void"]
        protos[m.group(2)] = (m.group(1).strip(), params)
    return protos


def c_offsets(struct, fields):
    src = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HDR}"', "int main(void) {",
           f'  printf("size %zu\\n", sizeof({struct}));']
    for f in fields:
        src.append(f'  printf("{f} %zu\\n", offsetof({struct}, {f}));')
    src.append("  return 0; }")
    with tempfile.TemporaryDirectory() as d:
        c, exe = os.path.join(d, "o.c"), os.path.join(d, "o")
        open(c, "w").write("\n".join(src))
        subprocess.run(["gcc", c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    return {k: int(v) for k, v in (ln.split() for ln in out.splitlines())}


@pytest.mark.parametrize("name", ["ndg_control", "ndg_thermo"])
def test_derived_types_match_c_structs(name):
    fields = fortran_types()[name]
    assert fields, name
    off, layout = 0, {}
    for kind, _, nm, n in fields:
        size = KIND[kind][0]
        off = (off + size - 1) // size * size  # natural alignment, as C lays it out
        layout[nm] = off
        off += size * n
    size = (off + 7) // 8 * 8
    got = c_offsets(name, [f[2] for f in fields])
    assert got.pop("size") == size
    assert got == layout


def test_interfaces_match_header_and_library():
    funcs = fortran_interfaces()
    protos = c_prototypes()
    L = ctypes.CDLL(LIB) if os.path.exists(LIB) else None
    assert len(funcs) >= 25
    for fname, f in funcs.items():
        cname = f["cname"]
        assert cname in protos, cname
        ret, params = protos[cname]
        assert (ret == "int") == (f["ret"] == "integer(c_int)"), cname
        assert (ret == "const char *") == (f["ret"] == "type(c_ptr)"), cname
        assert len(params) == len(f["args"]), cname
        for a, p in zip(f["args"], params):
            kind, value, n = f["decl"][a]
            c_ptr = "*" in p or p.split()[0].endswith("_cb")
            if value:
                # by value: a plain C scalar, or the pointer a c_ptr/c_funptr holds
                assert c_ptr == (kind in ("type(c_ptr)", "type(c_funptr)")), (cname, a, p)
                if kind == "integer(c_int)":
                    assert p.split()[0] == "int", (cname, a, p)
                if kind == "real(c_double)":
                    assert p.split()[0] == "double", (cname, a, p)
            else:
                # by reference: the C parameter is a pointer (to the pointee's type)
                assert "*" in p, (cname, a, p)
                base = p.replace("const", "").split("*")[0].split()[-1]
                want = {"real(c_double)": "double", "integer(c_int)": "int",
                        "type(c_ptr)": "ndg_ctx", "type(ndg_control)": "ndg_control",
                        "type(ndg_thermo)": "ndg_thermo"}[kind]
                assert base == want, (cname, a, p)
        if L is not None:
            assert hasattr(L, cname), cname


def test_patched_dynamics_uses_declared_functions():
    funcs = set(fortran_interfaces()) | {"ndg_message"}
    called = set(re.findall(r"\b(ndg_\w+)\s*\(", open(DYN).read()))
    called -= {"ndg_control", "ndg_thermo_line", "ndg_check"}
    assert called and called <= funcs, called - funcs
