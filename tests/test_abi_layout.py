"""The Python mirror agrees with include/tga.h byte for byte: every struct's size and field offsets
(measured by a C program compiled against the header), and every function's parameter count and
scalar types against the ctypes signatures the mirror sets.  Runs on the CPU (gcc only)."""
from __future__ import annotations

import ctypes as C
import re
import subprocess
from pathlib import Path

import compresstemporalgraph_b200 as tga

ROOT = Path(__file__).resolve().parents[1]

STRUCTS = {
    "tga_dataset_cfg": tga._Cfg,
    "tga_info": tga._Info,
    "tga_timing": tga._Timing,
    "tga_query": tga._Query,
    "tga_tune_result": tga._TuneResult,
    "tga_server_stats": tga._ServerStats,
    "tga_gen_params": tga._GenParams,
    "tga_gen_summary": tga._GenSummary,
    "tga_ref_depths": tga._RefDepths,
}


def _c_layout(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "tga.h"', "int main(void) {"]
    for cname, py in STRUCTS.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", f"-I{ROOT / 'include'}", str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr  # a field the mirror names but the header lacks fails here
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    got = {}
    for line in out.splitlines():
        cname, key, val = line.split()
        got[(cname, key)] = int(val)
    return got


def test_struct_sizes_and_offsets_match_header(tmp_path):
    got = _c_layout(tmp_path)
    for cname, py in STRUCTS.items():
        assert C.sizeof(py) == got[(cname, "size")], cname
        for field, _ in py._fields_:
            assert getattr(py, field).offset == got[(cname, field)], (cname, field)


def test_mirror_names_every_header_field():
    """Every field of each header struct appears in its ctypes mirror (the converse of the
    compile check above)."""
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "tga.h").read_text(), flags=re.S)
    for cname, py in STRUCTS.items():
        body = re.search(r"typedef struct \{([^{}]*)\}\s*" + cname + r"\s*;", text)
        assert body, cname
        fields = []
        for decl in body.group(1).split(";"):
            decl = decl.strip()
            if not decl:
                continue
            decl = re.sub(r"\[[^\]]*\]", "", decl)  # arrays: the name before the brackets
            head, *rest = decl.split(",")
            fields.append(re.findall(r"(\w+)\s*$", head)[0])
            fields += [r.strip().lstrip("*").strip() for r in rest]
        assert fields == [f for f, _ in py._fields_], cname


_SCALARS = {
    "int32_t": C.c_int32, "int64_t": C.c_int64, "uint32_t": C.c_uint32, "uint64_t": C.c_uint64,
    "int": C.c_int, "float": C.c_float, "double": C.c_double,
}


def _declarations():
    text = re.sub(r"/\*.*?\*/", "", (ROOT / "include" / "tga.h").read_text(), flags=re.S)
    decls = {}
    for m in re.finditer(r"\b(?:const\s+)?[\w]+\s*\*?\s*\b(tga_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", text):
        params = [p.strip() for p in m.group(2).replace("\n", " ").split(",") if p.strip()]
        if params == ["void"]:
            params = []
        decls[m.group(1)] = params
    return decls


def test_function_signatures_match_header():
    decls = _declarations()
    assert len(decls) >= 50
    lib = tga._lib
    for name, params in decls.items():
        fn = getattr(lib, name)
        args = fn.argtypes or []
        assert len(args) == len(params), (name, params, args)
        for p, a in zip(params, args):
            if "*" in p:
                # any pointer: void*, typed pointer or char*; a typed pointer to a scalar points to
                # a type of the same size
                assert a is C.c_void_p or a is C.c_char_p or issubclass(a, C._Pointer), (name, p, a)
                base = p.replace("const", "").split()[0].rstrip("*")
                if a is not C.c_void_p and a is not C.c_char_p and base in _SCALARS:
                    assert C.sizeof(a._type_) == C.sizeof(_SCALARS[base]), (name, p, a)
            else:
                ctype = p.replace("const", "").split()[0]
                assert ctype in _SCALARS, (name, p)
                assert C.sizeof(a) == C.sizeof(_SCALARS[ctype]), (name, p, a)
                is_float = ctype in ("float", "double")
                assert (a in (C.c_float, C.c_double)) == is_float, (name, p, a)
