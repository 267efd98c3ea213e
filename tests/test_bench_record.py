"""bench.py's record, checked without a GPU: the clock summary (throttle reasons decoded, medians
per quarter of a long run, the unsampled case) and the reference arm's JSON line, which times the
CPU oracle on a small room."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_clock_summary_reasons_and_quarters():
    import bench
    c = bench.Clocks(0)
    assert c.summary()["reasons"] == ["unsampled"]
    # 8 samples at the burst clock, then 8 under the power cap (clock-event reason bit 0x4)
    c.rows = [(1965.0, 1965.0, 700.0, 0)] * 8 + [(1900.0, 1965.0, 995.0, 0x4)] * 8
    s = c.summary(quarters=True)
    assert s["reasons"] == ["sw_power_cap"]
    assert s["samples"] == 16 and s["sm_mhz_min"] == 1900.0 and s["sm_max_mhz"] == 1965.0
    assert s["sm_mhz_by_quarter"] == [1965.0, 1965.0, 1900.0, 1900.0]
    assert s["power_w_by_quarter"] == [700.0, 700.0, 995.0, 995.0]
    assert "sm_mhz_by_quarter" not in c.summary()


def test_reference_arm_line():
    cmd = [sys.executable, "bench.py", "--impl", "reference", "--room", "64", "48", "40", "--steps", "2",
           "--warmup", "3"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] == 2 and line["warmup"] == 3
    assert line["e2e"] == {"value": line["value"], "unit": line["unit"], "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    cpu = line["cpu_baseline"]
    assert cpu["value"] == line["value"] and cpu["kind"] in ("port", "reference") and cpu["cores"] >= 1
