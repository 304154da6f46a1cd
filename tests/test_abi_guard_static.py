"""Every exported C-ABI entry point that does host-side work runs its body
through abi_guard (paintop_b200/csrc/abi_guard.h), so no C++ exception can
unwind into the caller. This reads the sources: each definition of a pt_*
function inside the library's C++ sources either begins with
`return abi_guard(` or is one of the listed accessors, which only read plain
fields or forward to a guarded entry point."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "paintop_b200", "csrc")
HEADER = os.path.join(ROOT, "include", "paintop_cuda.h")

# no allocation, no locking, no standard-library call that can throw
ACCESSORS = {
    "pt_ctx_create",         # nothrow new, CUDA runtime calls and getenv only
    "pt_status_str",
    "pt_ctx_last_error",
    "pt_ctx_stream",
    "pt_ctx_last_timing",
    "pt_ctx_last_transfer",
    "pt_ctx_last_config",
    "pt_tile_config_count",
    "pt_tile_config_info",
    "pt_unet_param_count",
    "pt_op_compute",         # forwards to pt_op_compute_ex
}


def _sources():
    for d, _, files in os.walk(CSRC):
        for f in files:
            if f.endswith((".cu", ".cpp")):
                yield os.path.join(d, f)


def _declared():
    text = open(HEADER).read()
    return set(re.findall(r"\b(pt_[a-z0-9_]+)\s*\(", text))


def _definitions():
    """{name: first statement of the body} for every pt_* function defined."""
    out = {}
    for path in _sources():
        s = open(path).read()
        for m in re.finditer(r"\b(pt_[a-z0-9_]+)\s*\(", s):
            name = m.group(1)
            i, depth = m.end() - 1, 0
            while True:  # the matching parenthesis of the parameter list
                c = s[i]
                depth += c == "("
                depth -= c == ")"
                i += 1
                if depth == 0:
                    break
            j = i
            while j < len(s) and s[j] in " \t\n":
                j += 1
            if j < len(s) and s[j] == "{":
                body = s[j + 1:].lstrip()
                out[name] = (path, body[:40])
    return out


def test_every_declared_entry_point_is_defined():
    defs = _definitions()
    missing = sorted(n for n in _declared() if n not in defs and not n.startswith("pt_status"))
    assert not missing, missing


def test_entry_points_with_host_work_are_guarded():
    defs = _definitions()
    unguarded = []
    for name in sorted(_declared()):
        if name in ACCESSORS or name not in defs:
            continue
        path, first = defs[name]
        if not first.startswith("return abi_guard("):
            unguarded.append((name, os.path.relpath(path, ROOT), first))
    assert not unguarded, unguarded
