"""CPU: the C-ABI library loads, exports every symbol include/*.h declares, and
the ctypes mirror has the C layout.  No compute calls (no GPU here)."""
import ctypes as C
import re
import subprocess
import textwrap
from pathlib import Path

import pytest

from logosq_b200 import _lib, abi

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions():
    names = []
    for h in HEADERS:
        txt = h.read_text()
        names += re.findall(r"^\s*(?:int|const char \*)\s*(lq_\w+)\s*\(", txt, flags=re.M)
    return names


def test_header_declares_functions():
    names = declared_functions()
    assert "lq_state_create" in names and "lq_apply_circuit" in names
    assert len(names) == len(set(names))


def test_library_exports_every_declared_symbol():
    from logosq_b200 import build
    so = build.build()
    lb = C.CDLL(str(so))
    missing = [n for n in declared_functions() if not hasattr(lb, n)]
    assert not missing, missing


def test_loader_prototypes_cover_header():
    missing = [n for n in declared_functions() if n not in _lib.exported_symbols()]
    assert not missing, missing


def test_struct_layout_matches_c(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(textwrap.dedent(f"""
        #include <stdio.h>
        #include <stddef.h>
        #include "{ROOT / 'include' / 'logosq_b200.h'}"
        int main(void) {{
            printf("%zu %zu %zu %zu %zu\\n", sizeof(lq_gate), offsetof(lq_gate, angle),
                   offsetof(lq_gate, m), sizeof(lq_pauli_term), sizeof(lq_vqe_instance));
            printf("%d %d %d %d\\n", LQ_GATE_MATRIX2, LQ_ERR_UNSUPPORTED, LQ_C64, LQ_FLAG_TEXTBOOK);
            return 0;
        }}"""))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = [int(x) for x in out[0].split()]
    assert sizes[0] == C.sizeof(abi.LqGate) == abi.GATE_DTYPE.itemsize
    assert sizes[1] == abi.LqGate.angle.offset
    assert sizes[2] == abi.LqGate.m.offset
    assert sizes[3] == C.sizeof(abi.LqPauliTerm) == abi.TERM_DTYPE.itemsize
    assert sizes[4] == C.sizeof(abi.LqVqeInstance)
    consts = [int(x) for x in out[1].split()]
    assert consts == [abi.MATRIX2, abi.LQ_ERR_UNSUPPORTED, abi.LQ_C64, abi.FLAG_TEXTBOOK]


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "LIB_PATH", tmp_path / "nope.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(_lib.LogosQError):
        _lib.lib()


def test_rust_binding_covers_header():
    """The logosq-cuda crate's raw binding (logosq-cuda/src/ffi.rs) declares
    every entry point the header declares."""
    text = (ROOT / "logosq-cuda" / "src" / "ffi.rs").read_text()
    bound = set(re.findall(r"pub fn (lq_\w+)\(", text))
    missing = [n for n in declared_functions() if n not in bound]
    assert not missing, missing
