"""The op report as the reference's evidence bundle would store it.

The reference serialises a ``Report`` with serde (field names as declared,
``None`` fields omitted, stop reasons in kebab-case:
crates/paintop-ir/src/resource.rs:1064-1194) and writes bundle artifacts
through its canonical JSON emitter (crates/paintop-ir/src/canonical.rs:74-220):
keys sorted by their UTF-8 bytes, no whitespace, the minimal RFC 8259 escape
set, integers without a decimal point, and every float in ryu's shortest
round-trip form with ``-0.0`` folded to ``0.0`` and integral floats keeping
``.0``. Its pipeline skips report exports today
(crates/paintop-cpu/src/pipeline.rs:316-320), so the convergence metrics of a
solve never reach the bundle; :func:`write_report` writes them as
``outputs/<name>.json`` beside the image exports.
"""
from __future__ import annotations

import json
import math
import os

STOP_REASONS = ("converged", "max-iterations", "stalled")


class _Float(float):
    """A JSON number that serde would have produced from an f64 (not an integer)."""


def report_value(report) -> dict:
    """The serde value of a :class:`paintop_b200.ops.Report` (resource.rs:1064-1113):
    the Poisson ops leave channel_stats empty and content_hash blank
    (poisson_blend.rs:581-593) and carry the SolverData (resource.rs:1130-1174)."""
    v = {"extent": {"width": int(report.width), "height": int(report.height)},
         "channels": int(report.channels), "channel_stats": [], "all_finite": bool(report.all_finite),
         "content_hash": ""}
    s = report.solver
    if s is not None:
        sd = {"kind": s.kind, "steps": int(s.steps), "stability_number": _Float(s.stability_number),
              "stability_limit": _Float(s.stability_limit), "stable": bool(s.stable),
              "residual_history": [_Float(x) for x in s.residual_history],
              "total_energy": _Float(s.total_energy)}
        # Option fields: omitted when None (skip_serializing_if = "Option::is_none")
        if s.iterations is not None:
            sd["iterations"] = int(s.iterations)
        if s.stop_reason is not None:
            sd["stop_reason"] = s.stop_reason if isinstance(s.stop_reason, str) else STOP_REASONS[s.stop_reason]
        if s.converged is not None:
            sd["converged"] = bool(s.converged)
        if s.tolerance is not None:
            sd["tolerance"] = _Float(s.tolerance)
        if s.final_residual is not None:
            sd["final_residual"] = _Float(s.final_residual)
        v["solver"] = sd
    return v


def format_f64(x: float) -> str:
    """ryu's shortest round-trip rendering of a finite f64 as serde_json prints it:
    the shortest digits d1..dn with value 0.d1..dn x 10^kk, written positionally
    with a '.0' for integers when -5 < kk <= 16, else as d1[.d2..dn]e<kk-1>."""
    if not math.isfinite(x):
        raise ValueError(f"non-finite float {x!r} cannot be canonicalised")
    if x == 0.0:
        return "0.0"
    sign = "-" if x < 0 else ""
    # Python's repr is also the shortest round-trip digit string
    r = repr(abs(x))
    if "e" in r:
        m, _, e = r.partition("e")
        digits, e10 = m.replace(".", ""), int(e) - (len(m.split(".")[1]) if "." in m else 0)
    else:
        ip, _, fp = r.partition(".")
        fp = fp.rstrip("0")
        digits, e10 = (ip + fp).lstrip("0"), -len(fp)
        if not digits:
            digits = "0"
    stripped = digits.rstrip("0")
    e10 += len(digits) - len(stripped)
    digits = stripped
    n = len(digits)
    kk = n + e10  # 10^(kk-1) <= |x| < 10^kk
    if 0 <= e10 and kk <= 16:
        body = digits + "0" * e10 + ".0"
    elif 0 < kk <= 16:
        body = digits[:kk] + "." + digits[kk:]
    elif -5 < kk <= 0:
        body = "0." + "0" * (-kk) + digits
    elif n == 1:
        body = f"{digits}e{kk - 1}"
    else:
        body = f"{digits[0]}.{digits[1:]}e{kk - 1}"
    return sign + body


def _string(s: str) -> str:
    out = ['"']
    short = {'"': '\\"', "\\": "\\\\", "\b": "\\b", "\t": "\\t", "\n": "\\n", "\f": "\\f", "\r": "\\r"}
    for ch in s:
        if ch in short:
            out.append(short[ch])
        elif ord(ch) < 0x20:
            out.append(f"\\u00{ord(ch):02x}")
        else:
            out.append(ch)
    out.append('"')
    return "".join(out)


def canonical(value) -> str:
    """to_canonical_string (canonical.rs:74-220) of a JSON value built from dicts,
    lists, str, bool, int and float (a float is always emitted as a float)."""
    if value is None:
        return "null"
    if value is True:
        return "true"
    if value is False:
        return "false"
    if isinstance(value, float):
        return format_f64(value)
    if isinstance(value, int):
        return str(value)
    if isinstance(value, str):
        return _string(value)
    if isinstance(value, (list, tuple)):
        return "[" + ",".join(canonical(v) for v in value) + "]"
    if isinstance(value, dict):
        keys = sorted(value, key=lambda k: k.encode("utf-8"))
        return "{" + ",".join(_string(k) + ":" + canonical(value[k]) for k in keys) + "}"
    raise TypeError(f"not a JSON value: {type(value).__name__}")


def report_json(report) -> str:
    """The canonical JSON bytes (as text) of an op report."""
    return canonical(report_value(report))


def write_report(bundle_dir: str, name: str, report) -> str:
    """Write `report` as ``outputs/<name>.json`` under a bundle directory; returns the
    bundle-relative path."""
    rel = os.path.join("outputs", f"{name}.json")
    path = os.path.join(bundle_dir, rel)
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w", encoding="utf-8") as f:
        f.write(report_json(report))
    os.replace(tmp, path)
    return rel


def parse(text: str):
    """Read canonical JSON back (floats stay floats, integers stay ints)."""
    return json.loads(text)
