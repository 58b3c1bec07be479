//! Links libappearance_cuda.so.  APPEARANCE_CUDA_LIB_DIR names the directory
//! that holds it (the in-tree build puts it in appearance_b200/); the CUDA
//! runtime comes from CUDA_HOME (default /usr/local/cuda).
use std::env;

fn main() {
    let lib_dir = env::var("APPEARANCE_CUDA_LIB_DIR").unwrap_or_else(|_| "../../appearance_b200".to_string());
    let cuda = env::var("CUDA_HOME").unwrap_or_else(|_| "/usr/local/cuda".to_string());
    println!("cargo:rustc-link-search=native={lib_dir}");
    println!("cargo:rustc-link-search=native={cuda}/lib64");
    println!("cargo:rustc-link-lib=dylib=appearance_cuda");
    println!("cargo:rustc-link-lib=dylib=cudart");
    println!("cargo:rerun-if-env-changed=APPEARANCE_CUDA_LIB_DIR");
    println!("cargo:rerun-if-env-changed=CUDA_HOME");
}
