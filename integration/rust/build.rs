// build.rs — compiles the B200 backend's CUDA sources with nvcc for sm_100a
// and links the resulting shared library into the turbogp crate.
//
// Not compiled here: this image has no Rust toolchain. The nvcc command lines
// are the ones turbogp_b200/build.py runs (and the repository's tests run),
// so the library this produces is the one the tests exercise.
//
// Inputs (environment):
//   TURBOGP_B200_SRC   path of the turbogp_b200 checkout (default ../turbogp_b200-repo)
//   NVCC               nvcc executable (default: nvcc on PATH, else /usr/local/cuda/bin/nvcc)
// The build only runs when the crate's `gpu-b200` feature is on.
use std::env;
use std::path::{Path, PathBuf};
use std::process::Command;

const SOURCES: [&str; 5] = ["scan_engine.cu", "aux_kernels.cu", "groupby_direct.cu", "capi.cu", "noalloc.cu"];

fn nvcc() -> PathBuf {
    if let Ok(p) = env::var("NVCC") {
        return PathBuf::from(p);
    }
    let on_path = Command::new("nvcc").arg("--version").output().map(|o| o.status.success()).unwrap_or(false);
    if on_path {
        PathBuf::from("nvcc")
    } else {
        PathBuf::from("/usr/local/cuda/bin/nvcc")
    }
}

fn run(cmd: &mut Command) {
    let status = cmd.status().unwrap_or_else(|e| panic!("could not start {:?}: {e}", cmd));
    assert!(status.success(), "{:?} failed with {status}", cmd);
}

fn main() {
    println!("cargo:rerun-if-env-changed=TURBOGP_B200_SRC");
    println!("cargo:rerun-if-env-changed=NVCC");
    if env::var_os("CARGO_FEATURE_GPU_B200").is_none() {
        return;
    }
    let root = PathBuf::from(env::var("TURBOGP_B200_SRC").unwrap_or_else(|_| "../turbogp_b200-repo".into()));
    let csrc = root.join("turbogp_b200").join("csrc");
    let include = root.join("include");
    let out = PathBuf::from(env::var("OUT_DIR").expect("cargo sets OUT_DIR"));
    let nvcc = nvcc();
    let arch = ["-gencode", "arch=compute_100a,code=sm_100a"];
    let mut objects = Vec::new();
    for src in SOURCES {
        let path = csrc.join(src);
        println!("cargo:rerun-if-changed={}", path.display());
        let obj = out.join(Path::new(src).with_extension("o"));
        run(Command::new(&nvcc)
            .args(arch)
            .args(["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden"])
            .arg("--diag-suppress=128,177")
            .arg(format!("-I{}", include.display()))
            .arg(format!("-I{}", csrc.display()))
            .arg("-c")
            .arg(&path)
            .arg("-o")
            .arg(&obj));
        objects.push(obj);
    }
    for header in ["device_common.cuh", "plan.hpp", "runtime.hpp"] {
        println!("cargo:rerun-if-changed={}", csrc.join(header).display());
    }
    println!("cargo:rerun-if-changed={}", include.join("turbogp_gpu.h").display());
    // One shared library with the CUDA runtime linked statically, as
    // turbogp_b200/build.py links it.
    let lib = out.join("libturbogp_b200.so");
    run(Command::new(&nvcc).args(arch).args(["-shared", "-cudart", "static", "-o"]).arg(&lib).args(&objects));
    println!("cargo:rustc-link-search=native={}", out.display());
    println!("cargo:rustc-link-lib=dylib=turbogp_b200");
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", out.display());
}
