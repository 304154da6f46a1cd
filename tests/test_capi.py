"""C-ABI tests that need no GPU: the library loads, exports every symbol the
header declares, reports a missing device as PT_NO_DEVICE, and the C++ host
layer validates op inputs and params with the reference's error classes,
codes and messages (crates/paintop-cpu/src/poisson_blend.rs:102-139,417-445,
603-632; screened_poisson.rs:66-123).
"""
import ctypes as C
import os
import re
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "paintop_cuda.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pt_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(cuda_lib):
    from paintop_b200 import _lib
    names = declared_symbols()
    assert len(names) >= 10
    for n in names:
        assert hasattr(cuda_lib, n), f"{n} missing from libpaintop_cuda.so"
    assert set(names) == set(_lib.EXPORTED)


def test_status_strings(cuda_lib):
    from paintop_b200 import _lib
    assert cuda_lib.pt_status_str(_lib.PT_OK) == b"ok"
    assert b"E_CUDA_UNAVAILABLE" in cuda_lib.pt_status_str(_lib.PT_NO_DEVICE)
    assert cuda_lib.pt_status_str(99) == b"unknown status"


def test_tile_configs(cuda_lib):
    n = cuda_lib.pt_tile_config_count()
    assert n >= 2
    for k in range(n):
        s, w, h = C.c_int32(), C.c_int32(), C.c_int32()
        assert cuda_lib.pt_tile_config_info(k, C.byref(s), C.byref(w), C.byref(h)) == 0
        assert 1 <= s.value <= 8 and w.value % 8 == 0 and h.value > 0
    assert cuda_lib.pt_tile_config_info(n, None, None, None) != 0


def _gpu_present():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_gpu_present(), reason="checks the no-device path")
def test_ctx_create_without_device_is_no_device(cuda_lib):
    from paintop_b200 import _lib
    h = C.c_void_p()
    assert cuda_lib.pt_ctx_create(0, C.byref(h)) == _lib.PT_NO_DEVICE
    assert not h.value


def test_injected_no_device_fault_in_child():
    # host fault injection: the library reports no device whatever the hardware
    code = ("import ctypes as C; from paintop_b200 import _lib; h=C.c_void_p(); "
            "import sys; sys.exit(_lib.lib().pt_ctx_create(0, C.byref(h)))")
    env = dict(os.environ, PAINTOP_CUDA_FAULT="no-device")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env)
    assert r.returncode == 1  # PT_NO_DEVICE


# ---- op validation through pt_op_compute with no device context -------------------

def _ports(names_kinds, w=8, h=8, c=1, mask_w=None, mask_h=None):
    from paintop_b200 import _lib
    ports = {}
    for name, kind in names_kinds:
        if kind == _lib.PT_KIND_MASK:
            mw, mh = mask_w or w, mask_h or h
            ports[name] = (kind, mw, mh, 1, np.zeros(mw * mh, np.float32))
        else:
            ports[name] = (kind, w, h, c, np.zeros(w * h * c, np.float32))
    return ports


def op_call(op_id, ports, params, solve_flags=None):
    from paintop_b200 import _lib
    L = _lib.lib()
    arr = (_lib.PtPort * len(ports))()
    keep = []
    out_n = 0
    for k, (name, (kind, w, h, c, s)) in enumerate(ports.items()):
        nm = name.encode()
        keep += [nm, s]
        arr[k] = _lib.PtPort(nm, kind, w, h, c, s.ctypes.data, s.size)
        if name in ("target", "anchor"):
            out_n = w * h * c
    cand = np.zeros(max(out_n, 1), np.float32)
    sd = _lib.PtSolverData()
    err = _lib.PtError()
    fin = C.c_int32()
    args = (None, op_id.encode(), arr, len(ports), params.encode(), cand.ctypes.data, out_n, C.byref(sd), None, 0,
            C.byref(fin), C.byref(err))
    st = L.pt_op_compute(*args) if solve_flags is None else L.pt_op_compute_ex(*args, solve_flags)
    return st, err.error_class.decode(), err.code.decode(), err.message.decode()


BLEND = "repair.poisson_blend@1"
SCREENED = "repair.screened_poisson@1"


def blend_ports(**kw):
    from paintop_b200 import _lib
    return _ports([("source", 0), ("target", 0), ("mask", _lib.PT_KIND_MASK)], **kw)


def screened_ports(**kw):
    from paintop_b200 import _lib
    return _ports([("guidance", 0), ("anchor", 0), ("mask", _lib.PT_KIND_MASK)], **kw)


@pytest.mark.parametrize("params,detail", [
    ('{"tolerance": 2.0}', "tolerance must be in (0, 1)"),
    ('{"tolerance": 0}', "tolerance must be in (0, 1)"),
    ('{"tolerance": "x"}', "tolerance must be a number"),
    ('{"max_iterations": 0}', "max_iterations must be in 1..=100000"),
    ('{"max_iterations": 100001}', "max_iterations must be in 1..=100000"),
    ('{"max_iterations": -3}', "max_iterations must be a positive integer"),
    ('{"max_iterations": 5.0}', "max_iterations must be a positive integer"),
    ('{"max_iterations": 5000000000}', "max_iterations must be a positive integer"),
])
def test_blend_param_errors(cuda_lib, params, detail):
    st, cls, code, msg = op_call(BLEND, blend_ports(), params)
    assert st == 2 and cls == "schema" and code == "E_POISSON_BLEND_PARAM"
    assert msg == "repair.poisson_blend: " + detail


@pytest.mark.parametrize("params,detail", [
    ('{"lambda": -1.0}', "lambda must be a finite value >= 0"),
    ('{"lambda": "big"}', "lambda must be a number"),
    ('{"lambda": 1, "tolerance": 1.5}', "tolerance must be in (0, 1)"),
])
def test_screened_param_errors(cuda_lib, params, detail):
    st, cls, code, msg = op_call(SCREENED, screened_ports(), params)
    assert st == 2 and cls == "schema" and code == "E_SCREENED_POISSON_PARAM"
    assert msg == "repair.screened_poisson: " + detail


def test_missing_port_is_a_reference_error(cuda_lib):
    from paintop_b200 import _lib
    ports = _ports([("source", 0), ("mask", _lib.PT_KIND_MASK)])
    st, cls, code, msg = op_call(BLEND, ports, "{}")
    assert (st, cls, code) == (2, "reference", "E_POISSON_BLEND_INPUT")
    assert msg == "repair.poisson_blend requires a `target` input value"


def test_wrong_kind_is_a_type_error(cuda_lib):
    ports = _ports([("source", 0), ("target", 0), ("mask", 0)])
    st, cls, code, msg = op_call(BLEND, ports, "{}")
    assert (cls, code) == ("type", "E_POISSON_BLEND_INPUT")
    assert msg == "repair.poisson_blend `mask` input must be a mask resource"


def test_mismatched_mask_extent_is_rejected(cuda_lib):
    # poisson_blend/tests.rs:258-266
    st, cls, code, msg = op_call(BLEND, blend_ports(mask_w=4, mask_h=4), "{}")
    assert (st, cls, code) == (2, "semantic", "E_POISSON_BLEND_SHAPE")
    assert msg == "repair.poisson_blend: the mask must share the images' extent"


def test_mismatched_layout_is_rejected(cuda_lib):
    from paintop_b200 import _lib
    ports = {"source": (0, 8, 8, 3, np.zeros(192, np.float32)),
             "target": (0, 8, 8, 4, np.zeros(256, np.float32)),
             "mask": (_lib.PT_KIND_MASK, 8, 8, 1, np.zeros(64, np.float32))}
    st, cls, code, msg = op_call(BLEND, ports, "{}")
    assert (cls, code) == ("semantic", "E_POISSON_BLEND_SHAPE")
    assert msg == "repair.poisson_blend: the source and target images must share a channel layout"


def test_screened_shape_errors_use_the_blend_shape_code(cuda_lib):
    st, cls, code, msg = op_call(SCREENED, screened_ports(mask_w=3, mask_h=8), "{}")
    assert (cls, code) == ("semantic", "E_POISSON_BLEND_SHAPE")
    assert msg.startswith("repair.screened_poisson: ")


def test_valid_request_without_device_is_policy_unavailable(cuda_lib):
    st, cls, code, _ = op_call(BLEND, blend_ports(), '{"tolerance": 1e-6, "max_iterations": 10}')
    assert (st, cls, code) == (1, "policy", "E_CUDA_UNAVAILABLE")


def test_params_validation_order_matches_reference(cuda_lib):
    # resolve_controls runs before the inputs are read (poisson_blend.rs:540-543)
    from paintop_b200 import _lib
    ports = _ports([("source", 0), ("mask", _lib.PT_KIND_MASK)])
    st, cls, code, _ = op_call(BLEND, ports, '{"tolerance": 5}')
    assert code == "E_POISSON_BLEND_PARAM"
    # screened reads lambda first (screened_poisson.rs:67-78)
    st, cls, code, msg = op_call(SCREENED, screened_ports(), '{"lambda": -2, "tolerance": 7}')
    assert msg.endswith("lambda must be a finite value >= 0")


def test_unknown_op_and_bad_json(cuda_lib):
    st, cls, code, _ = op_call("repair.nope@1", blend_ports(), "{}")
    assert st == 2 and cls == "reference"
    st, cls, code, _ = op_call(BLEND, blend_ports(), "{not json")
    assert st == 2 and cls == "parse"


def test_solve_flags_entry_point(cuda_lib):
    """pt_op_compute_ex, the entry point of the multigrid implementation: with
    flags 0 or PT_FLAG_MULTIGRID it validates exactly as pt_op_compute (the same
    errors, then no device); any other bit is refused before anything else."""
    from paintop_b200 import _lib
    for flags in (0, _lib.PT_FLAG_MULTIGRID):
        for params in ('{"tolerance": 2.0}', '{"max_iterations": 0}', "{not json"):
            assert op_call(BLEND, blend_ports(), params, flags) == op_call(BLEND, blend_ports(), params)
        assert op_call(SCREENED, screened_ports(mask_w=3, mask_h=8), "{}", flags) == \
            op_call(SCREENED, screened_ports(mask_w=3, mask_h=8), "{}")
        st, cls, code, _ = op_call(SCREENED, screened_ports(), '{"lambda": 0.5}', flags)
        assert (st, cls, code) == (1, "policy", "E_CUDA_UNAVAILABLE")
    for bad in (_lib.PT_FLAG_DEVICE_POINTERS, _lib.PT_FLAG_OMEGA_AUTO, _lib.PT_FLAG_MULTIGRID | 0x100):
        st, cls, code, msg = op_call(BLEND, blend_ports(), "{}", bad)
        assert (st, cls, code) == (2, "execution", "E_CUDA_SOLVE_FLAGS")
        assert msg == f"unsupported solve flags {bad}"
