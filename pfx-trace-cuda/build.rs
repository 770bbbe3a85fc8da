// Links libpfxtrace.so (built by pfx_b200/build.py).  PFXT_LIB_DIR names the
// directory that holds it; by default the library beside this crate.
fn main() {
    let dir = std::env::var("PFXT_LIB_DIR").unwrap_or_else(|_| {
        let here = std::env::var("CARGO_MANIFEST_DIR").expect("cargo sets CARGO_MANIFEST_DIR");
        format!("{here}/../pfx_b200/lib")
    });
    println!("cargo:rustc-link-search=native={dir}");
    println!("cargo:rustc-link-lib=dylib=pfxtrace");
    println!("cargo:rerun-if-env-changed=PFXT_LIB_DIR");
}
