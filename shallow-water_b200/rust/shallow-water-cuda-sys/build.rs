//! Links the prebuilt libswcuda.so (python shallow-water_b200/build.py).
//! SWCUDA_LIB_DIR names the directory that holds it; by default it is the
//! package directory two levels above this crate (shallow-water_b200/).
use std::env;
use std::path::PathBuf;

fn main() {
    let dir = match env::var("SWCUDA_LIB_DIR") {
        Ok(d) => PathBuf::from(d),
        Err(_) => PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap()).join("..").join(".."),
    };
    println!("cargo:rustc-link-search=native={}", dir.display());
    println!("cargo:rustc-link-lib=dylib=swcuda");
    println!("cargo:rerun-if-env-changed=SWCUDA_LIB_DIR");
    println!("cargo:rerun-if-changed={}", dir.join("libswcuda.so").display());
}
