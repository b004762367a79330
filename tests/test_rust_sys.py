"""The Rust -sys crate (ffi/cinder-cuda-sys) declares the C ABI of
include/cgs.h exactly: every exported function with the same name, number of
arguments, and per-argument kind (scalar / const pointer / mutable pointer,
plus the scalar's width), the same return kind, every #define constant, and
the #[repr(C)] structs with the header's fields in order. No Rust toolchain
is needed: both files are parsed as text."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cgs.h")
CRATE = os.path.join(ROOT, "ffi", "cinder-cuda-sys", "src", "lib.rs")

C_SCALARS = {"int": "i32", "int32_t": "i32", "uint32_t": "u32", "uint64_t": "u64",
             "float": "f32", "double": "f64", "uint8_t": "u8", "char": "i8", "void": "void",
             "size_t": "usize"}
RUST_SCALARS = {"c_int": "i32", "i32": "i32", "u32": "u32", "u64": "u64", "f32": "f32",
                "f64": "f64", "u8": "u8", "c_char": "i8", "c_void": "void", "usize": "usize"}


def _strip_c_comments(s):
    s = re.sub(r"/\*.*?\*/", " ", s, flags=re.S)
    return re.sub(r"//[^\n]*", " ", s)


def _c_kind(decl):
    """'const float* pos' -> ('cptr', 'f32'); 'uint32_t n' -> ('val', 'u32')."""
    decl = decl.strip()
    stars = decl.count("*")
    toks = decl.replace("*", " * ").split()
    const_first = toks[0] == "const"
    base = [t for t in toks if t not in ("const", "*")][0]
    base = C_SCALARS.get(base, base)
    if stars == 0:
        return ("val", base)
    if stars == 2:
        # T* const* (array of pointers) and T** (out pointer) are both
        # pointers to pointers; the outer constness decides
        outer_const = bool(re.search(r"\*\s*const\s*\*", decl))
        return ("cptr2" if outer_const else "mptr2", base)
    return ("cptr" if const_first else "mptr", base)


def _rust_kind(ty):
    ty = ty.strip()
    m = re.match(r"\*(const|mut)\s+\*(const|mut)\s+(\w+)$", ty)
    if m:
        return ("cptr2" if m.group(1) == "const" else "mptr2", RUST_SCALARS.get(m.group(3), m.group(3)))
    m = re.match(r"\*(const|mut)\s+(\w+)$", ty)
    if m:
        return ("cptr" if m.group(1) == "const" else "mptr", RUST_SCALARS.get(m.group(2), m.group(2)))
    return ("val", RUST_SCALARS.get(ty, ty))


def header_functions():
    src = _strip_c_comments(open(HEADER).read())
    out = {}
    for m in re.finditer(r"(?:^|\n)\s*(const\s+char\s*\*|int)\s+(cgs_\w+)\s*\(([^)]*)\)\s*;", src):
        ret, name, args = m.group(1), m.group(2), m.group(3).strip()
        kinds = [] if args in ("", "void") else [_c_kind(a) for a in args.split(",")]
        out[name] = (("cptr", "i8") if "char" in ret else ("val", "i32"), kinds)
    return out


def crate_functions():
    src = open(CRATE).read()
    block = src[src.index('extern "C" {'):]
    block = re.sub(r"//[^\n]*", " ", block)
    out = {}
    for m in re.finditer(r"pub fn (cgs_\w+)\s*\((.*?)\)\s*(?:->\s*([^;]+))?;", block, flags=re.S):
        name, args, ret = m.group(1), m.group(2), (m.group(3) or "").strip()
        args = [a for a in (x.strip() for x in args.split(",")) if a]
        kinds = [_rust_kind(a.split(":", 1)[1]) for a in args]
        out[name] = (_rust_kind(ret) if ret else ("val", "void"), kinds)
    return out


def test_every_header_function_is_declared_identically():
    h, r = header_functions(), crate_functions()
    assert len(h) >= 45, sorted(h)
    assert set(h) == set(r), (sorted(set(h) - set(r)), sorted(set(r) - set(h)))
    for name, (hret, hargs) in h.items():
        rret, rargs = r[name]
        assert hret == rret, (name, hret, rret)
        assert len(hargs) == len(rargs), (name, hargs, rargs)
        for i, (a, b) in enumerate(zip(hargs, rargs)):
            assert a[0] == b[0], (name, i, a, b)
            # pointers to a header struct are typed in Rust; the header's
            # `void*` camera/compositor slots do not occur
            assert a[1] == b[1], (name, i, a, b)


def test_constants_match():
    src = _strip_c_comments(open(HEADER).read())
    consts = dict(re.findall(r"#define\s+(CGS_\w+)\s+(-?\d+)", src))
    crate = open(CRATE).read()
    rc = dict(re.findall(r"pub const (CGS_\w+):\s*\w+\s*=\s*(-?\d+);", crate))
    assert consts and set(consts) == set(rc), (sorted(set(consts) - set(rc)),
                                              sorted(set(rc) - set(consts)))
    for k, v in consts.items():
        assert int(rc[k]) == int(v), k


def _header_structs():
    src = _strip_c_comments(open(HEADER).read())
    out = {}
    for m in re.finditer(r"typedef struct (cgs_\w+)\s*\{(.*?)\}\s*\w+;", src, flags=re.S):
        fields = []
        for stmt in m.group(2).split(";"):
            stmt = stmt.strip()
            if not stmt:
                continue
            toks = stmt.split()
            base = C_SCALARS.get(toks[0], toks[0])
            for decl in " ".join(toks[1:]).split(","):
                decl = decl.strip()
                am = re.match(r"(\w+)\[(\w+)\]", decl)
                if am:
                    fields.append((am.group(1), base, am.group(2)))
                else:
                    fields.append((decl, base, None))
        out[m.group(1)] = fields
    return out


def _crate_structs():
    src = open(CRATE).read()
    out = {}
    for m in re.finditer(r"pub struct (cgs_\w+)\s*\{(.*?)\n\}", src, flags=re.S):
        if m.group(1) == "cgs_ctx":
            continue
        fields = []
        for fm in re.finditer(r"pub (\w+):\s*([^,]+),", m.group(2)):
            ty = fm.group(2).strip()
            am = re.match(r"\[(\w+);\s*(\w+)\]", ty)
            if am:
                fields.append((fm.group(1), RUST_SCALARS.get(am.group(1), am.group(1)),
                               am.group(2)))
            else:
                fields.append((fm.group(1), RUST_SCALARS.get(ty, ty), None))
        out[m.group(1)] = fields
    return out


def test_structs_match_field_by_field():
    h, r = _header_structs(), _crate_structs()
    assert set(h) == set(r), (sorted(set(h) - set(r)), sorted(set(r) - set(h)))
    for name, hf in h.items():
        assert hf == r[name], (name, hf, r[name])


def test_crate_manifest_links_the_library():
    d = os.path.join(ROOT, "ffi", "cinder-cuda-sys")
    cargo = open(os.path.join(d, "Cargo.toml")).read()
    build = open(os.path.join(d, "build.rs")).read()
    assert 'links = "cindergs"' in cargo
    assert "rustc-link-lib=dylib=cindergs" in build
    assert 'mod pipeline' in open(CRATE).read()
    safe = open(os.path.join(d, "src", "pipeline.rs")).read()
    for fn in ("execute_frame_gpu", "readback_framebuffer_rgba8", "invalidate_stage3",
               "invalidate", "acquire"):
        assert f"fn {fn}" in safe, fn
