"""The Fortran replacement modules (s2dw_b200/fortran/*.f90) bind the C ABI
with ISO_C_BINDING interfaces.  No Fortran compiler exists here, so this
checks them against include/s2dw_cuda.h statically: every bind(C) name is an
exported symbol, the argument counts agree, an argument passed by VALUE is a
C scalar of the matching kind (c_int <-> int, c_double <-> double) and every
other argument is a C pointer (arrays, outputs, type(c_ptr) arrays for the
per-scale pointer lists, character strings)."""
import os
import re

import pytest

from s2dw_b200._lib import lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FORTRAN = [os.path.join(ROOT, "s2dw_b200", "fortran", f) for f in ("s2dw_core_mod.f90", "s2dw_fileio_mod.f90")]
HEADER = os.path.join(ROOT, "include", "s2dw_cuda.h")


def _fortran_interfaces(path):
    lines, cur = [], ""
    for raw in open(path):
        s = raw.split("!")[0].rstrip()
        if not s.strip():
            continue
        s = s.strip()
        if s.startswith("&"):
            s = s[1:].strip()
        if s.endswith("&"):
            cur += s[:-1] + " "
            continue
        lines.append(cur + s)
        cur = ""
    out = {}
    i = 0
    head = re.compile(r"function\s+(\w+)\s*\(([^)]*)\)\s*bind\s*\(\s*C\s*,\s*name\s*=\s*'(\w+)'\s*\)", re.I)
    while i < len(lines):
        m = head.search(lines[i])
        if not m:
            i += 1
            continue
        fname, args, sym = m.group(1), [a.strip().lower() for a in m.group(2).split(",") if a.strip()], m.group(3)
        decl = {}
        i += 1
        while not re.match(r"end\s+function", lines[i], re.I):
            if "::" in lines[i] and not lines[i].lower().startswith("import"):
                spec, names = lines[i].split("::", 1)
                attrs = spec.lower()
                for nm in re.split(r",(?![^(]*\))", names):
                    nm = nm.strip()
                    base = nm.split("(")[0].strip().lower()
                    decl[base] = {"value": "value" in attrs, "type": attrs.split(",")[0].strip(),
                                  "array": "(" in nm}
            i += 1
        out[sym] = (fname, args, decl)
    return out


def _c_prototypes():
    text = re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"\b(?:int|long long|const char\s*\*|void)\s+(s2dwc_\w+)\s*\(([^;]*?)\)\s*;", text, re.S):
        params = [p.strip() for p in m.group(2).split(",")] if m.group(2).strip() not in ("", "void") else []
        out[m.group(1)] = params
    return out


INTERFACES = {}
for _f in FORTRAN:
    for _sym, _v in _fortran_interfaces(_f).items():
        INTERFACES.setdefault(_sym, (os.path.basename(_f),) + _v)


def test_every_fortran_module_binds_something():
    assert len(INTERFACES) >= 20
    for f in FORTRAN:
        assert _fortran_interfaces(f), f


@pytest.mark.parametrize("sym", sorted(INTERFACES))
def test_fortran_interface_matches_header(sym):
    mod, fname, args, decl = INTERFACES[sym]
    protos = _c_prototypes()
    assert sym in protos, f"{mod}: {sym} is not declared in include/s2dw_cuda.h"
    assert hasattr(lib(), sym), f"{sym} is not exported by the library"
    params = protos[sym]
    assert len(params) == len(args), f"{mod} {fname}: {len(args)} arguments, C has {len(params)}"
    for a, p in zip(args, params):
        d = decl.get(a)
        assert d is not None, f"{mod} {fname}: argument {a} has no declaration"
        if "*" in p:
            assert not d["value"] or d["type"].startswith("type(c_ptr)"), f"{sym}: {a} must be by reference ({p})"
            if "char" in p:
                assert d["type"].startswith("character"), f"{sym}: {a} ({d['type']}) for {p}"
            elif "*const *" in p.replace(" ", "").replace("*const*", "*const *") or p.count("*") == 2:
                assert d["type"].startswith("type(c_ptr)") and d["array"], f"{sym}: {a} for {p}"
            elif p.startswith(("double", "const double")):
                assert d["type"].startswith(("real(c_double)", "complex(c_double_complex)")), f"{sym}: {a} for {p}"
            elif p.startswith(("int", "const int")):
                assert d["type"].startswith("integer(c_int)"), f"{sym}: {a} for {p}"
        else:
            assert d["value"], f"{sym}: {a} must be VALUE for the C scalar {p}"
            ctype = p.rsplit(" ", 1)[0].replace("const ", "").strip()
            want = {"int": "integer(c_int)", "double": "real(c_double)", "long long": "integer(c_long_long)"}[ctype]
            assert d["type"] == want, f"{sym}: {a} is {d['type']}, C has {p}"
