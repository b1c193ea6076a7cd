// Added to rsr's build.rs, after its `cc` step (build.rs:4-9): links the
// prebuilt B200 engine.  `python rsr_b200/csrc/build.py` in the engine's
// checkout builds rsr_b200/librsrgpu.so (nvcc, sm_100a); RSR_B200_DIR points
// at that directory.
fn link_rsr_b200() {
    let engine_dir = std::env::var("RSR_B200_DIR").unwrap_or_else(|_| "../rsr-b200/rsr_b200".into());
    println!("cargo:rustc-link-search=native={engine_dir}");
    println!("cargo:rustc-link-lib=dylib=rsrgpu");
    println!("cargo:rustc-link-arg=-Wl,-rpath,{engine_dir}");
    println!("cargo:rerun-if-env-changed=RSR_B200_DIR");
}
