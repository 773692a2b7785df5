//! Links libvxl_sph.so (the CUDA library; it links the CUDA runtime statically). Its folder
//! comes from VXL_SPH_LIB_DIR; without it the build fails with the instruction below, since
//! a silent fallback would only move the error to load time.
fn main() {
    println!("cargo:rerun-if-env-changed=VXL_SPH_LIB_DIR");
    let dir = std::env::var("VXL_SPH_LIB_DIR").unwrap_or_else(|_| {
        panic!("set VXL_SPH_LIB_DIR to the folder of libvxl_sph.so (build it with rust-wl_b200/vxl_sph/build.py)")
    });
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=vxl_sph");
}
