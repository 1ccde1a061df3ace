// Links the prebuilt libdynamis_cuda.so (built by dynamis_b200/build.py with nvcc for sm_100a).
// DYNAMIS_CUDA_LIB_DIR names the directory that holds it.
fn main() {
    let dir = std::env::var("DYNAMIS_CUDA_LIB_DIR").expect("DYNAMIS_CUDA_LIB_DIR: the directory of libdynamis_cuda.so");
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=dynamis_cuda");
    println!("cargo:rerun-if-env-changed=DYNAMIS_CUDA_LIB_DIR");
}
