//! Links libtmpm.so.  TMPM_LIB_DIR names the directory holding the built
//! library (`make -C tessera_b200/csrc` writes it to `tessera_b200/`); without
//! it the crate expects the library on the default linker path.
fn main() {
    println!("cargo:rerun-if-env-changed=TMPM_LIB_DIR");
    if let Ok(dir) = std::env::var("TMPM_LIB_DIR") {
        println!("cargo:rustc-link-search=native={dir}");
    }
    println!("cargo:rustc-link-lib=dylib=tmpm");
}
