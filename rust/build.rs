// The qvd crate's build script, extended to link libqvdgpu.so (built by
// `python -m qevedo_simulator_b200.build`; QVDGPU_DIR names its folder).
// Not compiled here: this image has no Rust toolchain (no cargo or rustc).
fn main() {
    if std::env::var_os("CARGO_FEATURE_GPU").is_some() {
        let dir = std::env::var("QVDGPU_DIR").unwrap_or_else(|_| "../qevedo_simulator_b200".to_string());
        println!("cargo:rustc-link-search=native={dir}");
        println!("cargo:rustc-link-lib=dylib=qvdgpu");
        println!("cargo:rerun-if-env-changed=QVDGPU_DIR");
    }
}
