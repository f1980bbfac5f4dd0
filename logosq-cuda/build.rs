//! Compiles the engine's hand-written CUDA sources (logosq_b200/csrc) for
//! sm_100a with nvcc and links the resulting shared library.  The source list
//! and flags are the ones `logosq_b200/build.py` uses, so the Rust and Python
//! front ends load the same native code.

use std::env;
use std::path::PathBuf;
use std::process::Command;

const SOURCES: &[&str] = &[
    "api_state.cu",
    "gates.cu",
    "fused.cu",
    "variational.cu",
    "profile.cu",
    "batch.cu",
    "tc.cu",
    "learned.cu",
    "noise.cu",
];

const NVCC_FLAGS: &[&str] = &[
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-O2",
    "--expt-relaxed-constexpr",
    "-rdc=false",
];

fn run(cmd: &mut Command) {
    let status = cmd.status().unwrap_or_else(|e| panic!("failed to start {:?}: {}", cmd, e));
    if !status.success() {
        panic!("{:?} exited with {}", cmd, status);
    }
}

fn main() {
    let manifest = PathBuf::from(env::var("CARGO_MANIFEST_DIR").expect("CARGO_MANIFEST_DIR"));
    let root = manifest.parent().expect("crate sits inside the engine repository").to_path_buf();
    let csrc = root.join("logosq_b200").join("csrc");
    let include = root.join("include");
    let out = PathBuf::from(env::var("OUT_DIR").expect("OUT_DIR"));
    let nvcc = env::var("NVCC").unwrap_or_else(|_| "/usr/local/cuda/bin/nvcc".to_string());

    let mut objs = Vec::new();
    for s in SOURCES {
        let src = csrc.join(s);
        let obj = out.join(s).with_extension("o");
        run(Command::new(&nvcc).args(NVCC_FLAGS).arg("-c").arg(&src).arg("-o").arg(&obj));
        println!("cargo:rerun-if-changed={}", src.display());
        objs.push(obj);
    }
    for dir in [&csrc, &include] {
        for entry in std::fs::read_dir(dir).expect("source directory").flatten() {
            let p = entry.path();
            if matches!(p.extension().and_then(|e| e.to_str()), Some("h" | "cuh")) {
                println!("cargo:rerun-if-changed={}", p.display());
            }
        }
    }

    let lib = out.join("liblogosq_b200.so");
    run(Command::new(&nvcc)
        .args(["-shared", "-gencode", "arch=compute_100a,code=sm_100a"])
        .args(&objs)
        .arg("-o")
        .arg(&lib)
        .args(["-lcudart_static", "-ldl", "-lrt", "-lpthread"]));

    println!("cargo:rustc-link-search=native={}", out.display());
    println!("cargo:rustc-link-lib=dylib=logosq_b200");
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", out.display());
    println!("cargo:rerun-if-env-changed=NVCC");
}
