"""The Rust FFI crate (rust/paintop-cuda) cannot be compiled in this environment
(no Rust toolchain), so its binding, src/ffi.rs, is checked against
include/paintop_cuda.h here: every struct of the header with the same fields in
the same order and the same C types, every function with the same parameter
names and types, and every constant with the header's value. The crate's two
OpImplementations and the patches that register them are checked for the
symbols they rely on."""
import os
import re

from tests.test_capi import ROOT

HEADER = os.path.join(ROOT, "include", "paintop_cuda.h")
CRATE = os.path.join(ROOT, "rust", "paintop-cuda")
FFI = os.path.join(CRATE, "src", "ffi.rs")
PATCHES = os.path.join(ROOT, "rust", "patches")

BASE = {"uint32_t": "u32", "int32_t": "i32", "uint64_t": "u64", "int64_t": "i64", "double": "f64",
        "float": "f32", "size_t": "usize", "char": "c_char", "int": "c_int", "void": "c_void"}
SAME = {"c_int": {"c_int", "i32"}, "pt_status": {"pt_status"}}


def c_source(keep_defines=False):
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    if keep_defines:
        return text
    return "\n".join(line for line in text.splitlines() if not line.lstrip().startswith("#"))


def rust_type(ctype: str) -> str:
    """A C type (as written in the header) in the Rust binding's spelling.
    qual[0] is the constness of the base type, qual[i] that of the i-th pointer
    object; the i-th pointer (counted from the base) points to an object whose
    constness is qual[i-1]."""
    toks = ctype.replace("*", " * ").split()
    toks = [t for t in toks if t != "struct"]
    base = [t for t in toks if t not in ("*", "const")]
    assert len(base) == 1, ctype
    quals = [False]
    for t in toks:
        if t == "*":
            quals.append(False)
        elif t == "const":
            quals[-1] = True
    stars = len(quals) - 1
    out = ""
    for i in range(stars, 0, -1):
        out += "*const " if quals[i - 1] else "*mut "
    return out + BASE.get(base[0], base[0])


def same(r: str, c: str) -> bool:
    r, c = r.replace(" ", ""), c.replace(" ", "")
    return r == c or r in SAME.get(c, ())


def c_structs():
    out = {}
    for name, body in re.findall(r"typedef struct (\w+) \{(.*?)\} \1;", c_source(), flags=re.S):
        fields = []
        for decl in body.split(";"):
            decl = " ".join(decl.split())
            if not decl:
                continue
            m = re.match(r"(.*?)(\w+)\[(\d+)\]$", decl)
            if m:  # char name[N]
                fields.append((m.group(2), f"[{BASE.get(m.group(1).strip(), m.group(1).strip())}; {m.group(3)}]"))
                continue
            m = re.match(r"(.*?)\s*(\*?)\s*(\w+(?:\s*,\s*\w+)*)$", decl)
            ctype = (m.group(1) + m.group(2)).strip()
            for n in m.group(3).split(","):  # uint32_t width, height, channels;
                fields.append((n.strip(), rust_type(ctype)))
        out[name] = fields
    return out


def c_functions():
    """name -> (return type, [(parameter name, type)]) in the Rust spelling."""
    out = {}
    for chunk in c_source().split(";"):
        decl = " ".join(re.split(r"[{}]", chunk)[-1].split())
        m = re.match(r"^(.*?)\b(pt_\w+)\s*\((.*)\)$", decl)
        if not m or m.group(1).startswith("typedef"):
            continue
        ps = []
        for p in m.group(3).split(","):
            p = p.strip()
            if p and p != "void":
                pm = re.match(r"(.*?)(\w+)$", p)
                ps.append((pm.group(2), rust_type(pm.group(1))))
        out[m.group(2)] = (rust_type(m.group(1)), ps)
    return out


def c_constants():
    out = {}
    for name, val in re.findall(r"#define (PT_[A-Z_0-9]+) (.+)", c_source(keep_defines=True)):
        v = val.strip()
        v = re.sub(r"(?<=[0-9a-fA-F])u\b", "", v)
        try:
            out[name] = int(eval(v, {}))
        except Exception:
            continue
    for name, val in re.findall(r"\b(PT_[A-Z_]+) = (\d+)", c_source()):
        out[name] = int(val)
    return out


def ffi_source():
    return open(FFI).read()


def test_rust_structs_match_the_header():
    src = ffi_source()
    cs = c_structs()
    seen = set()
    for name, body in re.findall(r"#\[repr\(C\)\] pub struct (pt_\w+) \{(.*?)\}", src, flags=re.S):
        if "_p:" in body:  # an opaque handle
            continue
        fields = [(n, " ".join(t.split())) for n, t in re.findall(r"pub (\w+): ([^,]+?)(?:,|$)", body.strip())]
        assert name in cs, name
        assert [f[0] for f in fields] == [f[0] for f in cs[name]], name
        for (n, rt), (_, ct) in zip(fields, cs[name]):
            assert same(rt, ct), (name, n, rt, ct)
        seen.add(name)
    assert seen == set(cs)


def test_rust_functions_match_the_header():
    src = ffi_source()
    cf = c_functions()
    seen = set()
    for name, params, ret in re.findall(r"pub fn (pt_\w+)\((.*?)\)\s*(?:->\s*([^;]+))?;", src, flags=re.S):
        assert name in cf, name
        cret, cps = cf[name]
        rps = [(n, " ".join(t.split())) for n, t in
               re.findall(r"(\w+):\s*([^,]+)", " ".join(params.split()))]
        assert [n for n, _ in rps] == [n for n, _ in cps], (name, rps, cps)
        for k, ((_, r), (_, c)) in enumerate(zip(rps, cps)):
            assert same(r, c), (name, k, r, c)
        if ret.strip():
            assert same(ret.strip(), cret), (name, ret, cret)
        seen.add(name)
    assert seen == set(cf), sorted(set(cf) - seen)


def test_rust_constants_match_the_header():
    src = ffi_source()
    cc = c_constants()
    rc = {n: int(eval(v.replace("_", ""), {})) for n, v in
          re.findall(r"pub const (PT_[A-Z_0-9]+): \w+ = ([0-9xX*+ a-fA-F_]+);", src)}
    assert set(rc) == set(cc), sorted(set(cc) ^ set(rc))
    for n, v in cc.items():
        assert rc[n] == v, (n, rc[n], v)


def test_crate_files_and_patches_are_complete():
    for f in ("Cargo.toml", "build.rs", "src/ffi.rs", "src/lib.rs", "src/mask.rs"):
        assert os.path.exists(os.path.join(CRATE, f)), f
    lib = open(os.path.join(CRATE, "src", "lib.rs")).read()
    mask = open(os.path.join(CRATE, "src", "mask.rs")).read()
    for sym in ("pt_op_compute_ex", "impl OpImplementation for CudaPoisson", "PT_FLAG_MULTIGRID"):
        assert sym in lib, sym
    assert "impl OpImplementation for CudaMask" in mask and "pt_op_compute" in mask
    # every ffi function the two implementations call is declared in ffi.rs
    declared = set(re.findall(r"pub fn (pt_\w+)\(", ffi_source()))
    for used in re.findall(r"ffi::(pt_\w+)\(", lib + mask):
        assert used in declared, used
    patches = {f: open(os.path.join(PATCHES, f)).read() for f in os.listdir(PATCHES)}
    joined = "\n".join(patches.values())
    assert 'ImplId::new("cuda", "poisson", 1)' in joined
    assert 'ImplId::new("cuda", "multigrid", 1)' in joined
    assert 'ImplId::new("cuda", "mask", 1)' in joined
    assert "allowed_backends" in joined and "write_json" in joined or "to_canonical_bytes" in joined
    for text in patches.values():  # unified diffs against the reference's own paths
        assert re.search(r"^--- a/crates/", text, flags=re.M) and re.search(r"^\+\+\+ b/crates/", text, flags=re.M)
        assert re.search(r"^@@ -\d+(,\d+)? \+\d+(,\d+)? @@", text, flags=re.M)
