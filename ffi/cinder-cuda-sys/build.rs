//! Links libcindergs.so, the library `python -m cindergs_b200.build` writes to
//! `cindergs_b200/_lib/` (nvcc, `-gencode arch=compute_100a,code=sm_100a`, the
//! CUDA runtime linked statically, so nothing else needs linking).
//! `CINDERGS_LIB_DIR` overrides the directory.
use std::env;
use std::path::PathBuf;

fn main() {
    let dir = match env::var("CINDERGS_LIB_DIR") {
        Ok(d) => PathBuf::from(d),
        Err(_) => {
            let manifest = PathBuf::from(env::var("CARGO_MANIFEST_DIR").expect("cargo sets it"));
            manifest.join("..").join("..").join("cindergs_b200").join("_lib")
        }
    };
    println!("cargo:rerun-if-env-changed=CINDERGS_LIB_DIR");
    println!("cargo:rerun-if-changed={}", dir.join("libcindergs.so").display());
    println!("cargo:rustc-link-search=native={}", dir.display());
    println!("cargo:rustc-link-lib=dylib=cindergs");
    // let binaries find the library next to where it was built
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", dir.display());
}
