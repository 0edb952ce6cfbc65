//! Links libmaille_gpu.so. MAILLE_GPU_LIB_DIR names the folder that holds it (the library is
//! built by `python -m maille_b200.build`, in-tree next to maille_b200/__init__.py); the CUDA
//! runtime is linked into it statically, so nothing else is needed at link time.
fn main() {
    let dir = std::env::var("MAILLE_GPU_LIB_DIR")
        .expect("set MAILLE_GPU_LIB_DIR to the folder holding libmaille_gpu.so");
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=maille_gpu");
    println!("cargo:rerun-if-env-changed=MAILLE_GPU_LIB_DIR");
}
