// Links libglc.so.  GLC_LIB_DIR names the directory that holds it; by default the in-tree build
// output (zksync-crypto-gpu_b200/_build, made by `python zksync-crypto-gpu_b200/build.py`).
use std::env;
use std::path::PathBuf;

fn main() {
    println!("cargo:rerun-if-env-changed=GLC_LIB_DIR");
    let dir = match env::var("GLC_LIB_DIR") {
        Ok(d) => PathBuf::from(d),
        Err(_) => PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap()).join("../../_build"),
    };
    println!("cargo:rustc-link-search=native={}", dir.display());
    println!("cargo:rustc-link-lib=dylib=glc");
    println!("cargo:rustc-link-arg=-Wl,-rpath,{}", dir.display());
}
