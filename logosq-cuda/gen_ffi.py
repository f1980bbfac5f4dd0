#!/usr/bin/env python3
"""Generate src/ffi.rs (the raw `extern "C"` block of the logosq-cuda crate)
from include/logosq_b200.h, the single source of truth of the C ABI.

    python logosq-cuda/gen_ffi.py          # rewrite src/ffi.rs
    python logosq-cuda/gen_ffi.py --check  # exit 1 if src/ffi.rs is stale

Every `int lq_*(...)` prototype, every enum constant and the three plain-data
structs of the header become Rust items; C types map one to one onto
`std::os::raw` / fixed-width Rust types, array parameters decay to pointers
as they do in C.
"""
from __future__ import annotations

import re
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
HEADER = HERE.parent / "include" / "logosq_b200.h"
OUT = HERE / "src" / "ffi.rs"

HANDLES = {"lq_state": "LqState", "lq_batch": "LqBatch", "lq_mlp": "LqMlp"}
STRUCTS = {"lq_gate": "LqGate", "lq_pauli_term": "LqPauliTerm",
           "lq_vqe_instance": "LqVqeInstance"}
SCALARS = {"int": "c_int", "unsigned": "c_uint", "int32_t": "i32", "int64_t": "i64",
           "uint64_t": "u64", "uint32_t": "u32", "size_t": "usize", "double": "f64",
           "float": "f32", "char": "c_char", "void": "c_void", "long long": "c_longlong"}


def strip_comments(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return re.sub(r"//[^\n]*", " ", text)


def rust_type(ctype: str) -> str:
    """C parameter or field type (without the name) -> Rust type."""
    t = ctype.replace("struct ", "").strip()
    const = t.startswith("const ")
    if const:
        t = t[len("const "):].strip()
    stars = t.count("*")
    base = t.replace("*", "").replace("const", "").strip()
    if base in HANDLES:
        rb = HANDLES[base]
    elif base in STRUCTS:
        rb = STRUCTS[base]
    elif base in SCALARS:
        rb = SCALARS[base]
    else:
        raise ValueError(f"unmapped C type {ctype!r}")
    if stars == 0:
        return rb
    out = rb
    for k in range(stars):
        # the outermost pointer carries the const of the pointee only for one level
        out = ("*const " if (const and k == 0) else "*mut ") + out
    return out


def split_param(p: str) -> tuple[str, str]:
    """'const double m[8]' -> ('const double *', 'm')."""
    p = p.strip()
    arr = re.search(r"\[[^\]]*\]\s*$", p)
    if arr:
        p = p[: arr.start()].strip()
    m = re.match(r"^(.*?)(\w+)$", p)
    ctype, name = m.group(1).strip(), m.group(2)
    if arr:
        ctype += " *"
    return ctype, name


def functions(src: str):
    out = []
    for name, params in re.findall(r"\bint\s+(lq_\w+)\s*\(([^;{]*?)\)\s*;", src, flags=re.S):
        ps = [q for q in (x.strip() for x in params.replace("\n", " ").split(",")) if q]
        if ps == ["void"]:
            ps = []
        out.append((name, "c_int", [split_param(q) for q in ps]))
    for rtype, name, params in re.findall(r"\b(const\s+char\s*\*)\s*(lq_\w+)\s*\(([^;{]*?)\)\s*;",
                                          src, flags=re.S):
        ps = [q for q in (x.strip() for x in params.replace("\n", " ").split(",")) if q]
        if ps == ["void"]:
            ps = []
        out.append((name, "*const c_char", [split_param(q) for q in ps]))
    return out


def enums(src: str):
    vals = []
    for body in re.findall(r"\benum\s*\{([^}]*)\}", src, flags=re.S):
        nxt = 0
        for item in body.split(","):
            item = item.strip()
            if not item:
                continue
            if "=" in item:
                k, v = (x.strip() for x in item.split("=", 1))
                nxt = int(v, 0)
            else:
                k = item
            vals.append((k, nxt))
            nxt += 1
    return vals


def structs(src: str):
    out = []
    for body, name in re.findall(r"typedef\s+struct\s+\w+\s*\{([^}]*)\}\s*(\w+)\s*;", src, flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            arr = re.search(r"\[(\d+)\]\s*$", decl)
            if arr:
                decl = decl[: arr.start()].strip()
            m = re.match(r"^(.*?)(\w+)$", decl)
            ctype, fname = m.group(1).strip(), m.group(2)
            rt = rust_type(ctype)
            if arr:
                rt = f"[{rt}; {arr.group(1)}]"
            fields.append((fname, rt))
        out.append((name, fields))
    return out


def render() -> str:
    src = strip_comments(HEADER.read_text())
    lines = [
        "// @generated by logosq-cuda/gen_ffi.py from include/logosq_b200.h -- do not edit.",
        "//! Raw bindings of the B200 engine's C ABI (`include/logosq_b200.h`).",
        "#![allow(non_camel_case_types, dead_code, clippy::missing_safety_doc)]",
        "",
        "use std::os::raw::{c_char, c_int, c_longlong, c_uint, c_void};",
        "",
    ]
    for k, v in enums(src):
        lines.append(f"pub const {k}: c_int = {v};")
    lines.append("")
    for h in HANDLES.values():
        lines.append("#[repr(C)]")
        lines.append(f"pub struct {h} {{\n    _opaque: [u8; 0],\n}}")
        lines.append("")
    for cname, fields in structs(src):
        rname = STRUCTS[cname]
        lines.append("#[repr(C)]")
        lines.append("#[derive(Clone, Copy, Debug)]")
        lines.append(f"pub struct {rname} {{")
        for fname, rt in fields:
            lines.append(f"    pub {fname}: {rt},")
        lines.append("}")
        lines.append("")
    lines.append('extern "C" {')
    for name, ret, params in functions(src):
        args = ", ".join(f"{pn}: {rust_type(pt)}" for pt, pn in params)
        lines.append(f"    pub fn {name}({args}) -> {ret};")
    lines.append("}")
    lines.append("")
    return "\n".join(lines)


def main() -> int:
    text = render()
    if "--check" in sys.argv:
        ok = OUT.exists() and OUT.read_text() == text
        if not ok:
            print(f"{OUT} is stale: run python logosq-cuda/gen_ffi.py", file=sys.stderr)
        return 0 if ok else 1
    OUT.write_text(text)
    return 0


if __name__ == "__main__":
    sys.exit(main())
