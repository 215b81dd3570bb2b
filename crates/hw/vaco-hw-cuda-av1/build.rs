//! Links the B200 post-filter library (`libvaco_av1_gpu.so`, built by
//! `python -m vaco_b200.build` with nvcc for sm_100a) and the CUDA runtime.
//!
//! `VACO_B200_LIB_DIR` names the directory holding the library;
//! `CUDA_HOME` (default /usr/local/cuda) the toolkit whose lib64 holds
//! libcudart.

fn main() {
    println!("cargo:rerun-if-env-changed=VACO_B200_LIB_DIR");
    println!("cargo:rerun-if-env-changed=CUDA_HOME");
    if let Ok(dir) = std::env::var("VACO_B200_LIB_DIR") {
        println!("cargo:rustc-link-search=native={dir}");
        println!("cargo:rustc-link-arg=-Wl,-rpath,{dir}");
    }
    let cuda = std::env::var("CUDA_HOME").unwrap_or_else(|_| String::from("/usr/local/cuda"));
    println!("cargo:rustc-link-search=native={cuda}/lib64");
    println!("cargo:rustc-link-lib=dylib=cudart");
}
