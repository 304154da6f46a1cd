//! Links the prebuilt libpaintop_cuda.so (built for sm_100a by
//! `python -m paintop_b200.build`; the CUDA runtime is linked into it
//! statically, so the only runtime dependency is the NVIDIA driver).
fn main() {
    let dir = std::env::var("PAINTOP_CUDA_LIB_DIR").unwrap_or_else(|_| "../../paintop_b200".into());
    println!("cargo:rerun-if-env-changed=PAINTOP_CUDA_LIB_DIR");
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=paintop_cuda");
}
