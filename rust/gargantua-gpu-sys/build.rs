// Links libgargantua_gpu.so: its directory comes from GARGANTUA_GPU_LIB_DIR
// (the gargantua_b200/ directory of this repository after
// `python -m gargantua_b200.build`).
fn main() {
    println!("cargo:rerun-if-env-changed=GARGANTUA_GPU_LIB_DIR");
    if let Ok(dir) = std::env::var("GARGANTUA_GPU_LIB_DIR") {
        println!("cargo:rustc-link-search=native={dir}");
    }
    println!("cargo:rustc-link-lib=dylib=gargantua_gpu");
}
