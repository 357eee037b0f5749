"""CPU tests of the config 3/4/5 legs that the default bench line carries: a
leg's JSON fields are kept, a leg that fails or runs too long becomes an
error entry, and the config-2 line is printed either way."""
import json
import subprocess
import sys

from conftest import ROOT

sys.path.insert(0, ROOT)


class _Done:
    def __init__(self, rc, out, err=""):
        self.returncode, self.stdout, self.stderr = rc, out, err


def test_legs_kept_failed_and_timed_out(monkeypatch):
    import bench
    calls = []

    def fake_run(cmd, capture_output, text, timeout):
        wk = cmd[cmd.index("--workload") + 1]
        calls.append((wk, timeout, cmd))
        if wk == "cfg3":
            line = {"metric": "m3", "value": 47.0, "unit": "BD steps/s", "config": {"workload": "w3"},
                    "clocks": {"sm_mhz": 1965.0}, "not_kept": 1}
            return _Done(0, "log line\n" + json.dumps(line) + "\n")
        if wk == "cfg4":
            return _Done(1, "", "Traceback: something broke")
        raise subprocess.TimeoutExpired(cmd, timeout)

    monkeypatch.setattr(subprocess, "run", fake_run)
    res = bench.run_other_configs()
    assert [c[0] for c in calls] == ["cfg3", "cfg4", "cfg5"]
    assert all("--no-other-configs" in c[2] for c in calls)
    assert res["cfg3"]["value"] == 47.0 and res["cfg3"]["config"] == "w3" and "not_kept" not in res["cfg3"]
    assert res["cfg4"]["error"].startswith("exit 1") and "something broke" in res["cfg4"]["error"]
    assert "did not finish" in res["cfg5"]["error"]
    assert all("wall_s" in v for v in res.values())
