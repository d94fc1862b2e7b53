"""CPU: bench.py's workload presets and overrides (--config, --n, --rc, --dist) and its modes."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def parse(monkeypatch, *argv):
    import bench

    monkeypatch.setattr(sys, "argv", ["bench.py", *argv])
    return bench, bench.parse()


def test_default_is_the_headline_workload(monkeypatch):
    bench, a = parse(monkeypatch)
    cfg = bench.workload(a)
    assert cfg == bench.CONFIGS["c2"]
    assert (a.mode, a.decomp, a.impl, a.gpus) == ("config", "replicas", "ours", 1)


def test_overrides_rename_the_workload(monkeypatch):
    bench, a = parse(monkeypatch, "--config", "c4", "--n", "1000000", "--rc", "0.03", "--dist", "shell")
    cfg = bench.workload(a)
    assert cfg["n"] == 1_000_000 and cfg["rc"] == 0.03 and cfg["dist"] == "sphere"
    assert cfg["lo"] == (-0.5,) * 3 and cfg["hi"] == (1.5,) * 3
    assert cfg["workload"] == "sphere-shell 1000000, rc=0.03"
    assert bench.CONFIGS["c4"]["n"] == 10_000_000       # the preset itself is untouched


def test_modes_and_decompositions_are_choices(monkeypatch):
    for m in ("config", "compat", "mixed"):
        _, a = parse(monkeypatch, "--mode", m)
        assert a.mode == m
    _, a = parse(monkeypatch, "--decomp", "slab")
    assert a.decomp == "slab"
    with pytest.raises(SystemExit):
        parse(monkeypatch, "--mode", "fp16")
