// Links the prebuilt librcmvs.so (built with `python -m rustcolmap_b200.build`,
// which compiles the CUDA sources for sm_100a with nvcc).  RCMVS_LIB_DIR names
// the folder that holds it; by default the package folder of this repository.
use std::env;
use std::path::PathBuf;

fn main() {
    let dir = match env::var("RCMVS_LIB_DIR") {
        Ok(d) => PathBuf::from(d),
        Err(_) => PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap())
            .join("..")
            .join("..")
            .join("rustcolmap_b200"),
    };
    println!("cargo:rustc-link-search=native={}", dir.display());
    println!("cargo:rustc-link-lib=dylib=rcmvs");
    // the library is found at run time through the same folder
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", dir.display());
    println!("cargo:rerun-if-env-changed=RCMVS_LIB_DIR");
    println!("cargo:rerun-if-changed=../../include/rcmvs.h");
}
