// Links liboxpt.so, built by oxideav-render-vulkan_b200/build.py (CUDA
// 12.9, sm_100a). OXPT_LIB_DIR names the directory that holds it.
fn main() {
    let dir = std::env::var("OXPT_LIB_DIR").unwrap_or_else(|_| "../../oxideav-render-vulkan_b200".into());
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=oxpt");
    println!("cargo:rerun-if-env-changed=OXPT_LIB_DIR");
}
