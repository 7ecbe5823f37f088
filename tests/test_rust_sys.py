"""The Rust binding crate (crates/tessera-mpm-cuda-sys) against include/tmpm.h.

cargo is not in this image, so the crate cannot be compiled here; this test
parses both files instead and checks that they describe the same ABI: every
#[repr(C)] struct has the header's fields in the same order with the
corresponding Rust types and array lengths, every header function is declared
in the extern "C" block with the same argument names and types and the same
return type (and nothing else is declared), and every enum constant has the
header's value.
"""

import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tmpm.h")
CRATE = os.path.join(ROOT, "crates", "tessera-mpm-cuda-sys")
LIB_RS = os.path.join(CRATE, "src", "lib.rs")

BASE = {
    "double": "f64", "float": "f32", "int32_t": "i32", "uint32_t": "u32", "uint64_t": "u64",
    "uint16_t": "u16", "uint8_t": "u8", "size_t": "usize", "char": "c_char", "void": "c_void",
}


def strip_comments(text):
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    return re.sub(r"//[^\n]*", " ", text)


def c_type_to_rust(decl: str, param: bool):
    """'const double *' / 'TmpmSession **' / 'double' -> Rust type string (no spaces)."""
    decl = decl.strip()
    stars = decl.count("*")
    const = decl.startswith("const ")
    base = decl.replace("const ", "").replace("*", "").strip()
    rust = BASE.get(base, base)
    if stars == 0:
        return "()" if rust == "c_void" and not param else rust
    out = rust
    for level in range(stars):
        # `const` qualifies the innermost pointee only
        out = ("*const" if (level == 0 and const) else "*mut") + out
    return out


def parse_header():
    text = strip_comments(open(HEADER).read())
    structs = {}
    for m in re.finditer(r"typedef\s+struct\s+(\w+)\s*\{(.*?)\}\s*(\w+)\s*;", text, flags=re.S):
        fields = []
        for line in m.group(2).split(";"):
            line = " ".join(line.split())
            if not line:
                continue
            fm = re.match(r"(.*?)(\w+)\s*(?:\[(\d+)\])?$", line)
            ctype, name, arr = fm.group(1), fm.group(2), fm.group(3)
            fields.append((name, c_type_to_rust(ctype, True), int(arr) if arr else None))
        structs[m.group(3)] = fields
    enums = {}
    for m in re.finditer(r"typedef\s+enum\s+\w+\s*\{(.*?)\}\s*\w+\s*;", text, flags=re.S):
        for item in m.group(1).split(","):
            item = item.strip()
            if item:
                k, v = item.split("=")
                enums[k.strip()] = int(v)
    funcs = {}
    body = re.sub(r"typedef[^;]*?\{.*?\}\s*\w+\s*;", " ", text, flags=re.S)
    for m in re.finditer(r"([\w\s\*]+?)\b(tmpm_\w+)\s*\(([^)]*)\)\s*;", body):
        ret = c_type_to_rust(m.group(1), False)
        params = []
        args = " ".join(m.group(3).split())
        if args and args != "void":
            for a in args.split(","):
                a = a.strip()
                am = re.match(r"(.*?)(\w+)\s*(\[\d+\])?$", a)
                ctype = am.group(1) + ("*" if am.group(3) else "")  # an array parameter is a pointer
                params.append((am.group(2), c_type_to_rust(ctype, True)))
        funcs[m.group(2)] = (params, ret)
    return structs, enums, funcs


def parse_rust():
    text = strip_comments(open(LIB_RS).read())
    structs = {}
    for m in re.finditer(r"#\[repr\(C\)\][^{;]*?pub\s+struct\s+(\w+)\s*\{(.*?)\}", text, flags=re.S):
        fields = []
        for line in m.group(2).split(","):
            line = " ".join(line.split())
            if not line or line.startswith("_private"):
                continue
            fm = re.match(r"pub\s+(\w+)\s*:\s*(.+)$", line)
            name, rtype = fm.group(1), fm.group(2).replace(" ", "")
            am = re.match(r"\[(.+);(\d+)\]$", rtype)
            fields.append((name, am.group(1), int(am.group(2))) if am else (name, rtype, None))
        structs[m.group(1)] = fields
    consts = {m.group(1): int(m.group(2)) for m in re.finditer(r"pub\s+const\s+(\w+)\s*:\s*\w+\s*=\s*(-?\d+)\s*;",
                                                                text)}
    block = re.search(r'extern\s+"C"\s*\{(.*)\n\}', text, flags=re.S).group(1)
    funcs = {}
    for m in re.finditer(r"pub\s+fn\s+(\w+)\s*\((.*?)\)\s*(->\s*([^;]+))?;", block, flags=re.S):
        params = []
        args = " ".join(m.group(2).split())
        for a in filter(None, (x.strip() for x in args.split(","))):
            n, t = a.split(":", 1)
            params.append((n.strip(), t.replace(" ", "")))
        ret = m.group(4).replace(" ", "") if m.group(4) else "()"
        funcs[m.group(1)] = (params, ret)
    return structs, consts, funcs


def test_crate_files_exist():
    for f in ("Cargo.toml", "build.rs", os.path.join("src", "lib.rs")):
        assert os.path.exists(os.path.join(CRATE, f)), f
    assert 'links = "tmpm"' in open(os.path.join(CRATE, "Cargo.toml")).read()
    assert "rustc-link-lib=dylib=tmpm" in open(os.path.join(CRATE, "build.rs")).read()


def test_structs_match_the_header_field_for_field():
    hs, _, _ = parse_header()
    rs, _, _ = parse_rust()
    assert set(hs) <= set(rs), set(hs) - set(rs)
    for name, fields in hs.items():
        assert rs[name] == fields, (name, fields, rs[name])


def test_enum_values_match():
    _, he, _ = parse_header()
    _, rc, _ = parse_rust()
    assert len(he) > 30
    for k, v in he.items():
        assert rc.get(k) == v, (k, v, rc.get(k))


def test_every_function_is_declared_with_the_same_signature():
    _, _, hf = parse_header()
    _, _, rf = parse_rust()
    assert len(hf) > 60
    assert set(hf) == set(rf), (set(hf) ^ set(rf))
    for name, (params, ret) in hf.items():
        rparams, rret = rf[name]
        ret = "TmpmStatus" if ret == "TmpmStatus" else ret
        assert rret == ret, (name, ret, rret)
        assert rparams == params, (name, params, rparams)


def test_header_functions_are_exported_by_the_library():
    """The library built in-tree exports every function the header declares."""
    import ctypes

    _, _, hf = parse_header()
    path = os.path.join(ROOT, "tessera_b200", "libtmpm.so")
    if not os.path.exists(path):
        import pytest

        pytest.skip("libtmpm.so not built")
    lib = ctypes.CDLL(path)
    missing = [n for n in hf if not hasattr(lib, n)]
    assert not missing, missing
