"""Report export: the op report in the reference's canonical JSON
(crates/paintop-ir/src/canonical.rs, whose own test vectors are restated here)
with the serde field set of Report / SolverData
(crates/paintop-ir/src/resource.rs:1064-1194)."""
import json
import math
import random

import pytest

from paintop_b200 import ops
from paintop_b200.report_json import canonical, format_f64, report_json, write_report


# ---- canonical.rs tests (:231-380) -----------------------------------------------
def test_sorts_object_keys_lexicographically():
    assert canonical({"z": 1, "a": 2, "m": 3}) == '{"a":2,"m":3,"z":1}'


def test_key_order_does_not_affect_output():
    assert canonical({"b": {"d": 1, "c": 2}, "a": [3, 2, 1]}) == canonical({"a": [3, 2, 1], "b": {"c": 2, "d": 1}})


def test_no_insignificant_whitespace_and_nested_sorting():
    assert canonical({"a": [1, 2, {"b": 3}], "c": "x"}) == '{"a":[1,2,{"b":3}],"c":"x"}'
    assert canonical({"outer": {"y": {"b": 1, "a": 2}, "x": 0}}) == '{"outer":{"x":0,"y":{"a":2,"b":1}}}'
    assert canonical([3, 1, 2, "z", "a"]) == '[3,1,2,"z","a"]'


def test_integers_and_integral_floats():
    assert [canonical(v) for v in (0, 8, -17, 12345678901234567890)] == ["0", "8", "-17", "12345678901234567890"]
    assert canonical(8.0) == "8.0" and canonical(8.0) != canonical(8)
    assert canonical(-0.0) == "0.0" == canonical(0.0)


def test_floats_round_trip_through_canonical_text():
    for raw in (0.1, 8.5, -3.25, 1e-300, 2.2250738585072014e-308, 123.456):
        assert float(canonical(raw)) == raw


def test_strings_escape_only_the_required_characters():
    assert canonical("a\"b\\c\n\t\r\b\f\x01") == "\"a\\\"b\\\\c\\n\\t\\r\\b\\f\\u0001\""
    s = "héllo — 世界 🎨"
    assert canonical(s).encode("utf-8") == ('"' + s + '"').encode("utf-8")
    assert canonical(None) == "null" and canonical(True) == "true" and canonical(False) == "false"
    assert canonical({}) == "{}" and canonical([]) == "[]"


def test_non_finite_floats_are_rejected():
    with pytest.raises(ValueError):
        canonical(float("nan"))
    with pytest.raises(ValueError):
        canonical(float("inf"))


# ---- ryu's layout (serde_json's f64 Display) -------------------------------------
@pytest.mark.parametrize("x,text", [
    (1e-7, "1e-7"), (1e-6, "1e-6"), (1e-5, "0.00001"), (0.0001, "0.0001"), (123.0, "123.0"),
    (1e15, "1000000000000000.0"), (1e16, "1e16"), (1.5e16, "1.5e16"), (1e21, "1e21"),
    (9.93920165187303e-07, "9.93920165187303e-7"), (3.0000000000000004e-05, "0.000030000000000000004"),
    (5e-324, "5e-324"), (1.7976931348623157e308, "1.7976931348623157e308"), (-2.5, "-2.5"), (100.0, "100.0"),
])
def test_float_layout(x, text):
    assert format_f64(x) == text


def test_float_text_is_shortest_and_round_trips():
    rng = random.Random(5)
    for _ in range(3000):
        x = rng.choice([rng.uniform(-1, 1), math.ldexp(rng.random(), rng.randint(-1070, 1023)),
                        float(rng.randint(-10**12, 10**12))])
        t = format_f64(x)
        assert float(t) == x
        digits = t.lstrip("-").split("e")[0].replace(".", "").strip("0")
        assert len(digits) <= len(repr(abs(x)).split("e")[0].replace(".", "").strip("0")) or x == 0.0


# ---- the report ---------------------------------------------------------------------
def _report(**over):
    sd = ops.SolverData(kind="screened-poisson", steps=3, stability_number=0.0, stability_limit=0.0, stable=True,
                        residual_history=[0.5, 0.01, 2e-7], total_energy=0.0, iterations=3,
                        stop_reason="converged", converged=True, tolerance=1e-6, final_residual=2e-7)
    for k, v in over.items():
        setattr(sd, k, v)
    return ops.Report(64, 32, 4, True, sd)


def test_report_serialises_like_serde():
    text = report_json(_report())
    assert text == (
        '{"all_finite":true,"channel_stats":[],"channels":4,"content_hash":"","extent":{"height":32,"width":64},'
        '"solver":{"converged":true,"final_residual":2e-7,"iterations":3,"kind":"screened-poisson",'
        '"residual_history":[0.5,0.01,2e-7],"stability_limit":0.0,"stability_number":0.0,"stable":true,'
        '"steps":3,"stop_reason":"converged","tolerance":1e-6,"total_energy":0.0}}')
    v = json.loads(text)
    assert len(v["solver"]["residual_history"]) == v["solver"]["iterations"]


def test_none_options_are_omitted_and_stop_reasons_are_kebab_case():
    v = json.loads(report_json(_report(iterations=None, converged=None, tolerance=None, final_residual=None,
                                       stop_reason="max-iterations")))
    assert set(v["solver"]) == {"kind", "steps", "stability_number", "stability_limit", "stable",
                                "residual_history", "total_energy", "stop_reason"}
    assert v["solver"]["stop_reason"] == "max-iterations"
    v = json.loads(report_json(ops.Report(8, 8, 1, False)))
    assert "solver" not in v and v["all_finite"] is False


def test_write_report_into_a_bundle(tmp_path):
    rel = write_report(str(tmp_path), "report", _report())
    assert rel == "outputs/report.json"
    assert (tmp_path / rel).read_text(encoding="utf-8") == _report().to_json()
