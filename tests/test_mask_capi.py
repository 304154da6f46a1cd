"""mask.ellipse@1 and mask.polygon@1 through pt_op_compute with no device
context: params are validated with the reference's error classes, codes and
messages (crates/paintop-cpu/src/ellipse.rs:119-159,221-297,506-540;
crates/paintop-cpu/src/mask_polygon.rs:90-152,427-452; the rejection tests of
ellipse/tests.rs:306-396 and mask_polygon/tests.rs:259-279), and a valid request
without a device is the Policy error E_CUDA_UNAVAILABLE."""
import ctypes as C

import numpy as np
import pytest

ELLIPSE = "mask.ellipse@1"
POLYGON = "mask.polygon@1"


def mask_call(op_id, params, w=8, h=8, ports=None, count=None, solve_flags=None):
    from paintop_b200 import _lib
    L = _lib.lib()
    ports = {"extent_from": (0, w, h, 3, np.zeros(w * h * 3, np.float32))} if ports is None else ports
    arr = (_lib.PtPort * max(1, len(ports)))()
    keep = []
    for k, (name, (kind, pw, ph, c, s)) in enumerate(ports.items()):
        nm = name.encode()
        keep += [nm, s]
        arr[k] = _lib.PtPort(nm, kind, pw, ph, c, s.ctypes.data, s.size)
    n = w * h if count is None else count
    out = np.zeros(max(n, 1), np.float32)
    err = _lib.PtError()
    args = (None, op_id.encode(), arr, len(ports), params.encode(), out.ctypes.data, n, None, None, 0, None,
            C.byref(err))
    st = L.pt_op_compute(*args) if solve_flags is None else L.pt_op_compute_ex(*args, solve_flags)
    return st, err.error_class.decode(), err.code.decode(), err.message.decode(), err.actual.decode()


@pytest.mark.parametrize("params,message", [
    ('{"radii_px": [3, 3]}', "mask.ellipse parameter `center_px`: missing required parameter"),
    ('{"center_px": 4, "radii_px": [3, 3]}', "mask.ellipse parameter `center_px`: must be a [x, y] array"),
    ('{"center_px": [4], "radii_px": [3, 3]}',
     "mask.ellipse parameter `center_px`: must have exactly two elements"),
    ('{"center_px": [4, "y"], "radii_px": [3, 3]}', "mask.ellipse parameter `center_px`: must be a number"),
    ('{"center_px": [4, 4]}', "mask.ellipse parameter `radii_px`: missing required parameter"),
    ('{"center_px": [4, 4], "radii_px": [0, 3]}',
     "mask.ellipse `radii_px.x` must be a strictly positive radius, got 0"),
    ('{"center_px": [4, 4], "radii_px": [3, -2.5]}',
     "mask.ellipse `radii_px.y` must be a strictly positive radius, got -2.5"),
    ('{"center_px": [4, 4], "radii_px": [-1e-7, 1]}',
     "mask.ellipse `radii_px.x` must be a strictly positive radius, got -0.0000001"),
    ('{"center_px": [4, 4], "radii_px": [-0.0, 1]}',
     "mask.ellipse `radii_px.x` must be a strictly positive radius, got -0"),
    ('{"center_px": [4, 4], "radii_px": [-1e21, 1]}',
     "mask.ellipse `radii_px.x` must be a strictly positive radius, got -1000000000000000000000"),
    ('{"center_px": [4, 4], "radii_px": [3, 3], "angle_rad": "x"}',
     "mask.ellipse parameter `angle_rad`: must be a number"),
    ('{"center_px": [4, 4], "radii_px": [3, 3], "antialias": 1}',
     "mask.ellipse parameter `antialias`: `antialias` must be a string"),
    ('{"center_px": [4, 4], "radii_px": [3, 3], "antialias": "msaa"}',
     "mask.ellipse only supports `antialias: analytic`, got `msaa`"),
    ('{"center_px": [4, 4], "radii_px": [3, 3], "edge": 2}',
     "mask.ellipse parameter `edge`: `edge` must be an object"),
    ('{"center_px": [4, 4], "radii_px": [3, 3], "edge": {"half_width_px": 1}}',
     "mask.ellipse parameter `edge.profile`: `edge.profile` must be a string"),
    ('{"center_px": [4, 4], "radii_px": [3, 3], "edge": {"profile": "linear", "half_width_px": 1}}',
     "mask.ellipse only supports `edge.profile: smoothstep`, got `linear`"),
    ('{"center_px": [4, 4], "radii_px": [3, 3], "edge": {"profile": "smoothstep"}}',
     "mask.ellipse parameter `edge.half_width_px`: `edge.half_width_px` is required"),
    ('{"center_px": [4, 4], "radii_px": [3, 3], "edge": {"profile": "smoothstep", "half_width_px": -1}}',
     "mask.ellipse parameter `edge.half_width_px`: must be non-negative"),
])
def test_ellipse_param_errors(cuda_lib, params, message):
    st, cls, code, msg, _ = mask_call(ELLIPSE, params)
    assert (st, cls, code) == (2, "schema", "E_ELLIPSE_PARAM")
    assert msg == message


@pytest.mark.parametrize("params,message", [
    ('{}', "mask.polygon requires a `points` array of [x, y] vertices"),
    ('{"points": "nope"}', "mask.polygon parameter: `points` must be an array of [x, y] pairs"),
    ('{"points": [[1, 2, 3]]}', "mask.polygon parameter: each vertex must have exactly two elements"),
    ('{"points": [5]}', "mask.polygon parameter: each vertex must be a [x, y] array"),
    ('{"points": [[1, "a"]]}', "mask.polygon parameter: coordinates must be numbers"),
    ('{"points": [[1, 1], [2, 2], [3, 3]], "fill_rule": "bogus"}',
     "mask.polygon `fill_rule` must be `nonzero` or `even-odd`"),
])
def test_polygon_param_errors(cuda_lib, params, message):
    st, cls, code, msg, _ = mask_call(POLYGON, params)
    assert (st, cls, code) == (2, "schema", "E_POLYGON_PARAM")
    assert msg == message


def test_missing_extent_is_a_reference_error(cuda_lib):
    st, cls, code, msg, _ = mask_call(ELLIPSE, '{"center_px": [1, 1], "radii_px": [1, 1]}', ports={})
    assert (st, cls, code) == (2, "reference", "E_ELLIPSE_INPUT")
    assert msg == "mask.ellipse requires an `extent_from` input value"
    st, cls, code, msg, _ = mask_call(POLYGON, "{}", ports={})
    assert (cls, code, msg) == ("reference", "E_POLYGON_INPUT", "mask.polygon requires an `extent_from` input value")


def test_extent_is_read_before_params(cuda_lib):
    # compute() takes the extent first (ellipse.rs:511-519, mask_polygon.rs:433-434)
    st, cls, code, _, _ = mask_call(POLYGON, '{"points": 1}', ports={})
    assert code == "E_POLYGON_INPUT"


def test_wrong_output_length_is_an_execution_error(cuda_lib):
    st, cls, code, msg, _ = mask_call(POLYGON, '{"points": [[0, 0], [4, 0], [0, 4]]}', count=7)
    assert (cls, code) == ("execution", "E_POLYGON_INPUT")
    assert msg == "mask.polygon produced a mask buffer of unexpected length 7"


def test_valid_requests_without_device_are_policy_unavailable(cuda_lib):
    for op, params in ((ELLIPSE, '{"center_px": [4, 4], "radii_px": [3, 2], "angle_rad": 0.5,'
                                 ' "antialias": "analytic", "edge": {"profile": "smoothstep", "half_width_px": 1}}'),
                       (POLYGON, '{"points": [[0, 0], [4, 0], [0, 4]], "fill_rule": "even-odd"}'),
                       (POLYGON, '{"points": [[0, 0]]}')):
        st, cls, code, _, _ = mask_call(op, params)
        assert (st, cls, code) == (1, "policy", "E_CUDA_UNAVAILABLE")


@pytest.mark.parametrize("op_id,params", [
    (ELLIPSE, '{"center_px": [4, 4], "radii_px": [3, 3]}'),
    (ELLIPSE, '{"center_px": [4, 4], "radii_px": [0, 3]}'),
    (POLYGON, '{"points": [[1, 1], [6, 1], [4, 6]]}'),
])
def test_mask_ops_ignore_the_multigrid_flag(cuda_lib, op_id, params):
    """pt_op_compute_ex: the mask generators ignore PT_FLAG_MULTIGRID (the
    same validation, then no device)."""
    from paintop_b200 import _lib
    assert mask_call(op_id, params, solve_flags=_lib.PT_FLAG_MULTIGRID) == mask_call(op_id, params)
