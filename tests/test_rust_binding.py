"""The Rust -sys crate (rust/rcmvs-sys) mirrors include/rcmvs.h: every
function with the same parameters, every struct with the same fields in the
same order, every constant with the same value.  No Rust toolchain exists
where this runs, so the crate is checked by parsing both sources, not by
compiling it."""
import os
import re

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "rcmvs.h")
CRATE = os.path.join(ROOT, "rust", "rcmvs-sys")

_BASE = {"int32_t": "i32", "int": "c_int", "uint32_t": "u32", "uint64_t": "u64", "double": "f64", "float": "f32",
         "uint8_t": "u8", "void": "c_void", "char": "c_char"}


def _rust_type(ctype):
    """C declaration type -> the Rust type the binding must use."""
    toks = ctype.replace("*", " * ").split()
    const = toks[0] == "const"
    i = 1 if const else 0
    out = _BASE.get(toks[i], toks[i])
    levels = []
    for t in toks[i + 1:]:
        if t == "*":
            levels.append(const)
            const = False
        elif t == "const":
            const = True
    for c in levels:
        out = ("*const " if c else "*mut ") + out
    return out


def _c_source():
    return re.sub(r"/\*.*?\*/", "", open(HEADER).read(), flags=re.S)


def _c_functions():
    out = {}
    for ret, name, args in re.findall(r"\n\s*((?:const\s+)?[\w\s\*]+?)\b(rcmvs_\w+)\s*\(([^;{]*?)\)\s*;", _c_source()):
        params = []
        if args.strip() and args.strip() != "void":
            for a in args.split(","):
                m = re.match(r"(.*?)(\w+)$", " ".join(a.split()))
                params.append(_rust_type(m.group(1)))
        out[name] = (params, None if ret.strip() == "void" else _rust_type(ret.strip()))
    return out


def _rust_source():
    return open(os.path.join(CRATE, "src", "lib.rs")).read()


def _rust_functions():
    src = _rust_source()
    block = src[src.index('extern "C" {'):]
    block = block[:block.index("\n}\n")]
    out = {}
    for name, args, ret in re.findall(r"pub fn (\w+)\(([^)]*)\)\s*(?:->\s*([^;]+))?;", block, flags=re.S):
        params = [" ".join(p.split(":", 1)[1].split()) for p in args.split(",") if p.strip()]
        out[name] = (params, ret.strip() if ret else None)
    return out


def test_every_function_has_the_same_signature():
    c, r = _c_functions(), _rust_functions()
    assert len(c) > 50
    assert sorted(c) == sorted(r)
    for name in c:
        assert c[name] == r[name], name


def _c_structs():
    out = {}
    for body, name in re.findall(r"typedef struct \w+ \{(.*?)\} (\w+);", _c_source(), flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            m = re.match(r"(.*?)([\w\s,\[\]0-9]+)$", decl)
            typ = decl.split()[0] if not decl.startswith("const") else " ".join(decl.split()[:2])
            rest = decl[len(typ):].strip()
            stars = len(rest) - len(rest.lstrip("*"))
            typ = typ + " *" * stars
            for f in rest.lstrip("*").split(","):
                f = f.strip().lstrip("*").strip()
                arr = re.match(r"(\w+)\[(\d+)\]", f)
                if arr:
                    fields.append((arr.group(1), f"[{_rust_type(typ)}; {arr.group(2)}]"))
                else:
                    fields.append((f, _rust_type(typ)))
            del m
        out[name] = fields
    return out


def _rust_structs():
    out = {}
    for name, body in re.findall(r"#\[repr\(C\)\]\s*(?:#\[derive[^\]]*\]\s*)?pub struct (\w+) \{(.*?)\n\}",
                                 _rust_source(), flags=re.S):
        if "_private" in body:
            continue
        out[name] = [(m[0], " ".join(m[1].split())) for m in re.findall(r"pub (\w+): ([^,\n]+),", body)]
    return out


def test_every_struct_has_the_same_fields():
    c, r = _c_structs(), _rust_structs()
    assert sorted(c) == sorted(r)
    for name in c:
        assert c[name] == r[name], name


def test_constants_match():
    src = open(HEADER).read()
    c = {k: int(v.rstrip("u")) for k, v in re.findall(r"#define (RCMVS_\w+) \(?(-?\d+u?)\)?", src)}
    r = {k: int(v) for k, v in re.findall(r"pub const (RCMVS_\w+): \w+ = (-?\d+);", _rust_source())}
    assert c and c == r


def test_crate_files_present():
    for f in ("Cargo.toml", "build.rs", "src/lib.rs"):
        assert os.path.exists(os.path.join(CRATE, f)), f
    assert 'links = "rcmvs"' in open(os.path.join(CRATE, "Cargo.toml")).read()
    assert "rustc-link-lib=dylib=rcmvs" in open(os.path.join(CRATE, "build.rs")).read()
