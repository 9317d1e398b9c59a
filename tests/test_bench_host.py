"""Host-side parts of bench.py (no GPU): the summaries of the other workloads
that the default single-GPU line carries, and that a workload whose run
fails is reported in the line instead of failing the bench."""
from __future__ import annotations

import json
import subprocess
import sys
from pathlib import Path

import bench

ROOT = Path(__file__).resolve().parents[1]


def test_summaries_keep_each_workloads_figures():
    c3 = {"metric": "Mcell-updates/s", "value": 37.5e3, "unit": "Mcell-updates/s", "ms_per_step": 1341.6,
          "roofline": {"frac": 0.50}, "e2e": {"value": 26.0e3}, "clocks": {"sm_mhz": 1965.0},
          "config": {"workload": "c3_128x128x512", "plan": "8,4,64,32,3,0,3"},
          "parity": {"spec_l2_max": 2.7e-5}, "fp64": {"value": 24.7e3}}
    s = bench._summary("c3", c3)
    assert (s["value"], s["frac"], s["e2e"], s["plan"], s["parity_spec_l2_max"], s["fp64"]) == \
        (37.5e3, 0.50, 26.0e3, "8,4,64,32,3,0,3", 2.7e-5, 24.7e3)
    c4 = {"metric": "Mcell-updates/s", "value": 28.0e3, "roofline": {"frac": 0.32}, "e2e": {"value": 26.1e3},
          "scenes_per_s": 73.6, "plain_one_at_a_time": {"scenes_per_s": 12.7, "speedup_batched": 5.8}}
    s = bench._summary("c4", c4)
    assert s["scenes_per_s"] == 73.6 and s["plain_one_at_a_time"]["speedup_batched"] == 5.8
    c5 = {"metric": "scenes/s", "value": 53.6, "speedup_vs_plain": 3.9, "accepted_scene_frac": 0.0,
          "transfer_rel_err": {"network_only_median": 0.60}}
    s = bench._summary("c5", c5)
    assert s["frac"] is None and s["e2e"] is None
    assert s["speedup_vs_plain"] == 3.9 and s["transfer_rel_err"]["network_only_median"] == 0.60
    json.dumps(s)  # the line stays plain JSON


def test_a_failing_workload_is_reported_not_fatal(monkeypatch):
    calls = []

    def fake_run(argv, **kw):
        calls.append((argv, kw.get("env", {})))
        if "c4" in argv:
            return subprocess.CompletedProcess(argv, 3, stdout="", stderr="no device\n")
        line = {"metric": "m", "value": 1.0, "unit": "u"}
        return subprocess.CompletedProcess(argv, 0, stdout="noise\n" + json.dumps(line) + "\n", stderr="")

    monkeypatch.setattr(bench.subprocess, "run", fake_run)
    monkeypatch.setenv("RANK", "0")
    monkeypatch.setenv("MASTER_PORT", "29500")
    res = bench.other_workloads()
    assert set(res) == {"c3", "c4", "c5"}
    assert res["c3"]["value"] == 1.0 and res["c5"]["value"] == 1.0
    assert "error" in res["c4"] and "exit 3" in res["c4"]["error"]
    for name in res:
        assert res[name]["command"].startswith("python bench.py --workload " + name)
    # every run is its own single-GPU process: no rendezvous variables
    for argv, env in calls:
        assert argv[0] == sys.executable and argv[1] == str(ROOT / "bench.py")
        assert "RANK" not in env and "MASTER_PORT" not in env
