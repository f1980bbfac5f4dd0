"""CPU: the logosq-cuda crate (the Rust front end a LogosQ user links) stays
consistent with the C ABI and with the Python build.

cargo and rustc are not installed here, so the crate is not compiled; these
checks keep its sources honest instead:
  * src/ffi.rs is exactly what gen_ffi.py generates from include/logosq_b200.h;
  * every header prototype has an `extern "C"` declaration with the same
    parameter names and mapped types, and every enum constant is bound;
  * build.rs compiles the same sources with the same nvcc flags as
    logosq_b200/build.py;
  * lib.rs calls only functions and constants the binding declares, and gives
    every gate struct of the reference's dense path a descriptor.
"""
import importlib.util
import re
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
CRATE = ROOT / "logosq-cuda"


def gen():
    spec = importlib.util.spec_from_file_location("gen_ffi", CRATE / "gen_ffi.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def rust_fns():
    text = (CRATE / "src" / "ffi.rs").read_text()
    out = {}
    for name, args, ret in re.findall(r"pub fn (lq_\w+)\((.*?)\) -> ([^;]+);", text):
        ps = [a.strip() for a in args.split(",") if a.strip()]
        out[name] = ([tuple(x.strip() for x in p.split(":", 1)) for p in ps], ret.strip())
    return out


def test_ffi_is_generated_from_header():
    r = subprocess.run([sys.executable, str(CRATE / "gen_ffi.py"), "--check"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_every_prototype_bound_with_matching_types():
    g = gen()
    src = g.strip_comments(g.HEADER.read_text())
    fns = g.functions(src)
    assert len(fns) > 60
    bound = rust_fns()
    for name, ret, params in fns:
        assert name in bound, name
        rparams, rret = bound[name]
        assert rret == ret, (name, rret, ret)
        assert [p[0] for p in rparams] == [pn for _, pn in params], name
        assert [p[1] for p in rparams] == [g.rust_type(pt) for pt, _ in params], name


def test_type_mapping_examples():
    g = gen()
    assert g.rust_type("const lq_state *") == "*const LqState"
    assert g.rust_type("lq_batch **") == "*mut *mut LqBatch"
    assert g.rust_type("double *") == "*mut f64"
    assert g.rust_type("const double *") == "*const f64"
    assert g.rust_type("uint64_t") == "u64"
    assert g.split_param("const double m[8]") == ("const double *", "m")


def test_constants_and_structs_bound():
    g = gen()
    src = g.strip_comments(g.HEADER.read_text())
    text = (CRATE / "src" / "ffi.rs").read_text()
    for k, v in g.enums(src):
        assert f"pub const {k}: c_int = {v};" in text, k
    for rname in ("LqGate", "LqPauliTerm", "LqVqeInstance", "LqState", "LqBatch", "LqMlp"):
        assert re.search(rf"pub struct {rname} \{{", text), rname
    assert text.count("#[repr(C)]") == 6


def test_build_rs_matches_python_build():
    from logosq_b200 import build as b
    rs = (CRATE / "build.rs").read_text()
    srcs = re.findall(r'"(\w+\.cu)"', rs[rs.index("const SOURCES"):rs.index("const NVCC_FLAGS")])
    assert srcs == b.SOURCES
    flags_block = rs[rs.index("const NVCC_FLAGS"):rs.index("fn run")]
    flags = re.findall(r'"([^"]+)"', flags_block)
    assert flags == b.NVCC_FLAGS
    assert "cargo:rustc-link-lib=dylib=logosq_b200" in rs


def test_lib_rs_uses_only_bound_items():
    lib = (CRATE / "src" / "lib.rs").read_text()
    ffi = (CRATE / "src" / "ffi.rs").read_text()
    fns = set(rust_fns())
    for name in set(re.findall(r"ffi::(lq_\w+)\(", lib)):
        assert name in fns, name
    for const in set(re.findall(r"ffi::(LQ_\w+)", lib)):
        assert f"pub const {const}:" in ffi, const
    # every gate struct of the dense path gets a descriptor
    for gate in ("HGate", "XGate", "YGate", "ZGate", "SGate", "TGate", "RXGate", "RYGate",
                 "RZGate", "PhaseGate", "U3Gate", "CNOTGate", "SWAPGate", "CZGate", "CPhaseGate",
                 "ToffoliGate", "CRXGate", "CRYGate", "CRZGate", "CPhaseParamGate", "RXXGate",
                 "RYYGate", "RZZGate"):
        assert re.search(rf"(impl GpuGate for {gate}\b|!\({gate},)", lib), gate
    assert "impl QuantumStateBackend for CudaState" in lib
