// Links libwavecore_b200.so. Its directory comes from WAVECORE_B200_LIB_DIR, or defaults to the
// in-tree build output (`python -m wavesim_b200.build` writes wavesim_b200/libwavecore_b200.so
// at the root of this repository).
use std::env;
use std::path::PathBuf;

fn main() {
    let dir = match env::var("WAVECORE_B200_LIB_DIR") {
        Ok(d) => PathBuf::from(d),
        Err(_) => PathBuf::from(env::var("CARGO_MANIFEST_DIR").unwrap()).join("../../wavesim_b200"),
    };
    println!("cargo:rerun-if-env-changed=WAVECORE_B200_LIB_DIR");
    println!("cargo:rerun-if-changed=../../include/wavecore_c.h");
    println!("cargo:rustc-link-search=native={}", dir.display());
    println!("cargo:rustc-link-lib=dylib=wavecore_b200");
}
