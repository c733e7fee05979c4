// Links libks_b200.so (built by `make -C atomic-sandbox_b200`) and the CUDA runtime it uses.
// KS_B200_ROOT: the directory holding this repository's atomic-sandbox_b200/.
fn main() {
    let root = std::env::var("KS_B200_ROOT").expect("set KS_B200_ROOT to the repository holding atomic-sandbox_b200/");
    println!("cargo:rustc-link-search=native={}/atomic-sandbox_b200", root);
    println!("cargo:rustc-link-lib=dylib=ks_b200");
    println!("cargo:rustc-link-lib=dylib=cudart");
    println!("cargo:rerun-if-env-changed=KS_B200_ROOT");
}
