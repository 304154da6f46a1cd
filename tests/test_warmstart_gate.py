"""The learned warm start's cost gate (paintop_b200.warmstart.GuessGate): the
network's guess is used only for shapes and methods whose measured time with
the guess (inference + warm-started solve) beat the plain solve's; any other
shape gets the plain solve. CPU only: the decision reads a fixed table."""
import json

import pytest


def test_gate_keys_follow_shape_and_method():
    from paintop_b200 import warmstart as w
    assert w.gate_key(4096, 4096, 3, 1, "sor") == "25:24:0:sor"
    assert w.gate_key(4096, 4096, 3, 1, "multigrid") == "25:24:0:multigrid"
    assert w.gate_key(256, 256, 1, 256, "sor") == "24:16:1:sor"
    with pytest.raises(ValueError):
        w.gate_key(8, 8, 1, 1, "jacobi")


def test_gate_uses_the_guess_only_where_it_was_measured_to_pay():
    from paintop_b200 import warmstart as w
    gate = w.GuessGate()
    table = json.load(open(w.GATE_TABLE))["entries"]
    assert table, "the committed gate table is empty"
    for e in table:
        lt, ll, batch, method = e["key"].split(":")
        assert method in w.METHODS and e["plain_ms"] > 0 and e["learned_ms"] > 0
        assert gate.entries[e["key"]] == e
    # the 4096^2 workload: the guess pays under SOR, not under multigrid
    assert gate.decide(4096, 4096, 3, 1, "sor")[0] is True
    assert gate.decide(4096, 4096, 3, 1, "multigrid")[0] is False
    # a batch of 256 small images: inference costs more than the sweeps it saves
    assert gate.decide(256, 256, 1, 256, "sor")[0] is False
    # a shape that was never measured: plain solve, no entry
    assert gate.decide(300, 200, 3, 1, "sor") == (False, None)


def test_gate_is_deterministic_and_reads_only_its_table(tmp_path):
    from paintop_b200 import warmstart as w
    p = tmp_path / "gate.json"
    p.write_text(json.dumps({"entries": [{"key": w.gate_key(640, 480, 3, 1, "sor"),
                                          "plain_ms": 10.0, "learned_ms": 9.0}]}))
    g = w.GuessGate(str(p))
    assert [g.decide(640, 480, 3)[0] for _ in range(3)] == [True] * 3
    assert g.decide(640, 480, 3, method="multigrid") == (False, None)
    assert w.GuessGate(str(tmp_path / "absent.json")).entries == {}
