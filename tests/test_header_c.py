"""include/paintop_cuda.h as a C consumer sees it (cgo, a Rust -sys crate, a C
host): it compiles as strict C99, every function it declares links against
libpaintop_cuda.so, and the structs have the layout the ctypes bindings in
paintop_b200/_lib.py assume. No GPU is needed."""
import ctypes
import os
import shutil
import subprocess

import pytest

from tests.test_capi import ROOT, declared_symbols

GCC = shutil.which("gcc")
pytestmark = pytest.mark.skipif(GCC is None, reason="no C compiler")
INCLUDE = os.path.join(ROOT, "include")
FLAGS = ["-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror", "-x", "c", "-", "-I", INCLUDE]

# C field -> ctypes field, per struct (the ctypes names avoid the keyword `lambda`)
STRUCTS = {
    "pt_problem": ("PtProblem", ["width", "height", "channels", "source_or_guidance", "target_or_anchor", "mask",
                                 ("lambda", "lambda_"), "max_iterations", "tolerance", "omega", "flags",
                                 "initial_guess"]),
    "pt_report": ("PtReport", ["iterations", "converged", "stop_reason", "tolerance", "final_residual",
                               "history_len", "omega_used", "refinements", "channel", "initial_residual",
                               "warm_start"]),
    "pt_port": ("PtPort", ["name", "kind", "width", "height", "channels", "samples", "sample_count"]),
    "pt_error": ("PtError", ["error_class", "code", "message", "actual"]),
    "pt_solver_data": ("PtSolverData", ["kind", "steps", "stability_number", "stability_limit", "stable",
                                        "total_energy", "iterations", "stop_reason", "converged", "tolerance",
                                        "final_residual", "history_len"]),
}


def test_header_is_c99_and_every_function_links(cuda_lib):
    names = declared_symbols()
    src = ['#include "paintop_cuda.h"', "#include <stdio.h>", "typedef void (*any_fn)(void);",
           "static any_fn const fns[] = {"]
    src += [f"  (any_fn)&{n}," for n in names]  # every symbol's address: the link must resolve each
    src += ["};", "int main(void) {", '  printf("%d\\n", (int)(sizeof fns / sizeof fns[0]));', "  return 0;", "}"]
    lib_dir = os.path.join(ROOT, "paintop_b200")
    r = subprocess.run([GCC] + FLAGS + ["-L", lib_dir, "-lpaintop_cuda", "-o", os.devnull],
                       input="\n".join(src), capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-3000:]


def test_struct_layouts_match_the_python_bindings():
    from paintop_b200 import _lib
    src = ['#include "paintop_cuda.h"', "#include <stddef.h>", "#include <stdio.h>", "int main(void) {"]
    for cname, (_, fields) in STRUCTS.items():
        src.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in fields:
            cf = f[0] if isinstance(f, tuple) else f
            src.append(f'  printf("{cname} {cf} %zu\\n", offsetof({cname}, {cf}));')
    src += ["  return 0;", "}"]
    build = os.path.join(ROOT, "paintop_b200", "_build")
    os.makedirs(build, exist_ok=True)
    exe = os.path.join(build, "header_layout")
    r = subprocess.run([GCC] + FLAGS + ["-o", exe], input="\n".join(src), capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([exe], capture_output=True, text=True, timeout=60, check=True).stdout.split("\n")
    got = {tuple(line.split()[:2]): int(line.split()[2]) for line in out if line.strip()}
    for cname, (pyname, fields) in STRUCTS.items():
        cls = getattr(_lib, pyname)
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for f in fields:
            cf, pf = f if isinstance(f, tuple) else (f, f)
            assert got[(cname, cf)] == getattr(cls, pf).offset, (cname, cf)
        # the bindings name exactly the header's fields, in order
        assert [f[1] if isinstance(f, tuple) else f for f in fields] == [n for n, _ in cls._fields_]
