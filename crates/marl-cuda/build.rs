//! Links libmarl_cuda.so, built by `python marl-ochre_b200/build.py` (nvcc,
//! sm_100a).  MARL_CUDA_LIB_DIR names the directory that holds it.
fn main() {
    let dir = std::env::var("MARL_CUDA_LIB_DIR")
        .expect("set MARL_CUDA_LIB_DIR to the directory of libmarl_cuda.so");
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=marl_cuda");
    println!("cargo:rerun-if-env-changed=MARL_CUDA_LIB_DIR");
}
