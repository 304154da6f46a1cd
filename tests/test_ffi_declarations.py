"""The Rust FFI crate written out in INTEGRATION.md cannot be compiled in this
environment (no Rust toolchain), so its `#[repr(C)]` structs and `extern "C"`
functions are checked against include/paintop_cuda.h here: the same fields in
the same order with the same C types, and the same parameter lists."""
import os
import re

from tests.test_capi import ROOT

HEADER = os.path.join(ROOT, "include", "paintop_cuda.h")
GUIDE = os.path.join(ROOT, "INTEGRATION.md")

BASE = {"uint32_t": "u32", "int32_t": "i32", "uint64_t": "u64", "int64_t": "i64", "double": "f64",
        "float": "f32", "size_t": "usize", "char": "c_char", "int": "c_int", "void": "c_void"}
SAME = {"c_int": {"c_int", "i32"}, "pt_status": {"pt_status", "i32", "c_int"}}


def c_source():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return "\n".join(line for line in text.splitlines() if not line.lstrip().startswith("#"))


def rust_type(ctype: str) -> str:
    """A C type (as written in the header) in the Rust binding's spelling."""
    toks = ctype.replace("*", " * ").split()
    stars = toks.count("*")
    const = "const" in toks
    base = [t for t in toks if t not in ("*", "const", "struct")]
    assert len(base) == 1, ctype
    b = BASE.get(base[0], base[0])
    if stars == 0:
        return b
    if stars == 1:
        return ("*const " if const else "*mut ") + b
    return "*mut " * stars + b


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
    """name -> (return type, [parameter types]) in the Rust spelling."""
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
                ps.append(rust_type(re.match(r"(.*?)(\w+)$", p).group(1)))
        out[m.group(2)] = (rust_type(m.group(1)), ps)
    return out


def rust_blocks():
    text = open(GUIDE).read()
    return "\n".join(re.findall(r"```rust\n(.*?)```", text, flags=re.S))


def test_rust_structs_match_the_header():
    src = rust_blocks()
    cs = c_structs()
    seen = 0
    for name, body in re.findall(r"#\[repr\(C\)\] pub struct (pt_\w+) \{(.*?)\}", src, flags=re.S):
        if "_p:" in body:  # an opaque handle
            continue
        fields = [(n, " ".join(t.split())) for n, t in re.findall(r"pub (\w+): ([^,]+?)(?:,|$)", body.strip())]
        assert name in cs, name
        assert [f[0] for f in fields] == [f[0] for f in cs[name]], name
        for (n, rt), (_, ct) in zip(fields, cs[name]):
            assert same(rt, ct), (name, n, rt, ct)
        seen += 1
    assert seen >= 3


def test_rust_functions_match_the_header():
    src = rust_blocks()
    cf = c_functions()
    seen = 0
    for name, params, ret in re.findall(r"pub fn (pt_\w+)\((.*?)\)\s*(?:->\s*([^;]+))?;", src, flags=re.S):
        assert name in cf, name
        cret, cps = cf[name]
        rps = [" ".join(t.split()) for t in re.findall(r"\w+:\s*([^,]+)", " ".join(params.split()))]
        assert len(rps) == len(cps), (name, rps, cps)
        for k, (r, c) in enumerate(zip(rps, cps)):
            assert same(r, c), (name, k, r, c)
        if ret.strip():
            assert same(ret.strip(), cret), (name, ret, cret)
        seen += 1
    assert seen >= 8
