//! Builds the device library from mesh_to_sdf_b200/csrc with nvcc for sm_100a
//! and links it statically (CUDA runtime included).  NOT COMPILED HERE: see
//! Cargo.toml.
//!
//! M2S_ROOT: the checkout of this repository (default: two directories up).
//! NVCC: the nvcc to use (default: nvcc on PATH, then /usr/local/cuda/bin/nvcc).
use std::env;
use std::path::{Path, PathBuf};
use std::process::Command;

fn nvcc() -> PathBuf {
    if let Ok(p) = env::var("NVCC") {
        return PathBuf::from(p);
    }
    let on_path = Command::new("nvcc").arg("--version").output().map(|o| o.status.success()).unwrap_or(false);
    if on_path { PathBuf::from("nvcc") } else { PathBuf::from("/usr/local/cuda/bin/nvcc") }
}

fn main() {
    let manifest = PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap());
    let root = env::var("M2S_ROOT").map(PathBuf::from).unwrap_or_else(|_| manifest.join("../.."));
    let csrc = root.join("mesh_to_sdf_b200").join("csrc");
    let include = root.join("include");
    let out = PathBuf::from(env::var("OUT_DIR").unwrap());
    let nvcc = nvcc();

    let mut objects = Vec::new();
    let mut sources: Vec<PathBuf> = std::fs::read_dir(&csrc)
        .expect("mesh_to_sdf_b200/csrc")
        .map(|e| e.unwrap().path())
        .filter(|p| p.extension().map_or(false, |x| x == "cu"))
        .collect();
    sources.sort();
    for src in &sources {
        let obj = out.join(format!("{}.o", src.file_name().unwrap().to_string_lossy()));
        // The same flags as mesh_to_sdf_b200/build.py (strict build: every
        // distance operation rounds like the reference).
        let ok = Command::new(&nvcc)
            .args(["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-lineinfo"])
            .args(["-Xcompiler", "-fPIC", "-I"])
            .arg(&include)
            .arg("-c")
            .arg(src)
            .arg("-o")
            .arg(&obj)
            .status()
            .expect("running nvcc")
            .success();
        assert!(ok, "nvcc failed on {}", src.display());
        objects.push(obj);
        println!("cargo:rerun-if-changed={}", src.display());
    }
    // Device link step for the relocatable pieces, then one static archive.
    let lib = out.join("libm2s.a");
    let ok = Command::new(&nvcc)
        .args(["-gencode", "arch=compute_100a,code=sm_100a", "-lib", "-o"])
        .arg(&lib)
        .args(&objects)
        .status()
        .expect("running nvcc -lib")
        .success();
    assert!(ok, "nvcc -lib failed");
    println!("cargo:rustc-link-search=native={}", out.display());
    println!("cargo:rustc-link-lib=static=m2s");
    let cuda_lib = env::var("CUDA_LIB").unwrap_or_else(|_| "/usr/local/cuda/lib64".to_string());
    if Path::new(&cuda_lib).exists() {
        println!("cargo:rustc-link-search=native={cuda_lib}");
    }
    println!("cargo:rustc-link-lib=static=cudart_static");
    for l in ["stdc++", "dl", "rt", "pthread"] {
        println!("cargo:rustc-link-lib=dylib={l}");
    }
    println!("cargo:rerun-if-changed={}", include.join("m2s.h").display());
    println!("cargo:rerun-if-env-changed=M2S_ROOT");
}
