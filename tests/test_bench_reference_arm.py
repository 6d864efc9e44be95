"""bench.py's reference arm on CPU: the JSON line carries the contract's keys and
describes its own bounded sample (a small beach here, to keep the test short)."""
import io
import json
from contextlib import redirect_stdout

import pytest

from oracle.refio import harness_available


@pytest.mark.skipif(not harness_available(), reason="reference harness not built")
def test_reference_arm_json_line(monkeypatch):
    import bench
    monkeypatch.setattr(bench, "SAMPLE_NX", 40)
    monkeypatch.setattr(bench, "SAMPLE_NY", 10)
    args = type("A", (), {"warmup": 1, "steps": 2, "gpus": 1})()
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(args, 1, 0, None)
    lines = [ln for ln in buf.getvalue().splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    out = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in out, key
    assert out["impl"] == "reference" and out["metric"] == bench.METRIC and out["unit"] == bench.UNIT
    assert out["value"] > 0 and out["steps"] == 2 and out["warmup"] == 1
    assert out["cpu_baseline"]["value"] == out["value"] and out["cpu_baseline"]["cores"] == 1
    assert out["cpu_baseline"]["kind"] == "reference" and "steps 2..3" in out["cpu_baseline"]["sample"]
    assert "lower bound" in out["cpu_baseline"]["sample"]
    assert out["e2e"] == {"value": out["value"], "unit": out["unit"], "h2d_bytes_per_step": 0,
                          "d2h_bytes_per_step": 0}
