// Links libcintx_cuda.so.  CINTX_CUDA_LIB_DIR names the folder that holds it (the library is
// built in-tree as cintx_b200/libcintx_cuda.so); without it the system search path is used.
fn main() {
    println!("cargo:rerun-if-env-changed=CINTX_CUDA_LIB_DIR");
    if let Ok(dir) = std::env::var("CINTX_CUDA_LIB_DIR") {
        println!("cargo:rustc-link-search=native={dir}");
        println!("cargo:rustc-link-arg=-Wl,-rpath,{dir}");
    }
    println!("cargo:rustc-link-lib=dylib=cintx_cuda");
}
