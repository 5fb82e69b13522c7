//! Builds libsrcuda.so with nvcc (sm_100a) from a checkout of this repository and
//! links it.  SRCUDA_DIR points at the checkout (the directory holding
//! `include/srcuda.h`); by default it is two levels above this crate.
use std::{env, path::PathBuf, process::Command};

fn main() {
    let dir = env::var_os("SRCUDA_DIR").map(PathBuf::from).unwrap_or_else(|| {
        PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap()).join("..").join("..")
    });
    let status = Command::new(env::var("PYTHON").unwrap_or_else(|_| "python3".to_owned()))
        .args(["-m", "spatialrust_b200.csrc.build"])
        .current_dir(&dir)
        .status()
        .expect("running the nvcc build of libsrcuda.so");
    assert!(status.success(), "the nvcc build of libsrcuda.so failed");
    let lib_dir = dir.join("spatialrust_b200");
    println!("cargo:rustc-link-search=native={}", lib_dir.display());
    println!("cargo:rustc-link-lib=dylib=srcuda");
    // the consumer finds the library at run time next to its binary or through this path
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", lib_dir.display());
    println!("cargo:rerun-if-changed={}", dir.join("include").join("srcuda.h").display());
    println!("cargo:rerun-if-changed={}", dir.join("spatialrust_b200").join("csrc").display());
    println!("cargo:rerun-if-env-changed=SRCUDA_DIR");
}
